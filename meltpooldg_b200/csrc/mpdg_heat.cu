// Handle, setup kernels, Krylov drivers and the C ABI of the B200-native heat
// operator (include/mpdg_heat.h).
//
// Everything a solve touches stays resident on the device: the geometry
// factors, the solution history, the inverse diagonal and its FP32 copy, the
// FP32 copies of the linearisation point and the Krylov vectors. Krylov
// scalars (alpha, beta, residual norms, convergence flag) are computed on the
// device by the last CTA of each fused reduction and every kernel of an
// iteration exits immediately once the flag is set, so the host only polls
// the flag every few iterations instead of synchronising per iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <array>
#include <vector>

#include "../../include/mpdg_heat.h"
#include "cell_args.cuh"
#include "degree_table.hpp"
#include "fe_tables.hpp"
#include "material_law.cuh"
#include "picard_tc_layout.hpp"
#include "reduce.cuh"
#include "source_eval.cuh"

using namespace mpdg;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const std::string &msg)
{
  g_err = msg;
  return code;
}

#define CU(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(e_ == cudaErrorMemoryAllocation ? MPDG_ERR_OUT_OF_MEMORY : MPDG_ERR_CUDA, \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

#define TRY(call)                  \
  do {                             \
    int r_ = (call);               \
    if (r_ != MPDG_OK) return r_;  \
  } while (0)

extern "C" const char *mpdg_last_error(void) { return g_err.c_str(); }

// the library's other translation units report errors through the same thread-local message
int mpdg_internal_fail(int code, const char *msg) { return fail(code, msg); }

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
constexpr int VT = 256;  // threads of the vector kernels

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

// one level of the FP32 p-multigrid hierarchy (level 0 is the solver's own handle)
struct MGLevel {
  mpdg_heat *h = nullptr;
  bool own = false;
  int ratio = 1;                        // node ratio of the transfer to the next coarser level
  float xi[8] = {0};                    // fine-cell node positions of that transfer, in [0, 1]
  float *b = nullptr, *x = nullptr, *d = nullptr, *Ax = nullptr;
  double *Tl = nullptr, *To = nullptr;  // injected linearisation point (levels > 0)
  double theta = 1.0, delta = 1.0;      // smoothing interval (centre, half width)
  int pre = 0, post = 0;                // Chebyshev steps before / after the coarse correction
                                        // (post: after the restart step; coarsest: pre only)
  std::vector<float> c1, c2;
};

struct mpdg_heat {
  int device = 0, sm_count = 148;
  cudaStream_t stream = nullptr;
  mpdg_mesh_desc desc{};
  int p = 1, n = 2, npt = 8;
  int64_t n_dofs = 0, n_cells = 0;
  MeshDims dims{};
  int geo = 0;  // 0 uniform box, 1 per-quadrature-point factors
  double hcell[3] = {1, 1, 1};
  DegreeTable tab;
  // geometry
  double *vert = nullptr;  // vertices (deformed meshes)
  double *geoq = nullptr;  // [cell][7][npt]
  float *geoq_f = nullptr;
  // coefficients
  mpdg_material mat{};
  int law = 0, need_told = 0;
  double latent = 0.0;  // latent heat of fusion (mpdg_heat_set_latent_heat)
  int acap = MPDG_APPARENT_QLQ;
  double dt = 0.0;
  const double *T_lin = nullptr, *T_old = nullptr;
  float *T_lin_f = nullptr, *T_old_f = nullptr;
  bool lin_f_dirty = true;
  // preconditioner
  double *inv_diag = nullptr;
  float *inv_diag_f = nullptr;
  bool diag_valid = false, diag_f_dirty = true;
  double eig_min = 0.0, eig_max = 0.0;
  bool eig_valid = false;
  float *kq = nullptr;  // FP32 conductivity at the q-points (Picard preconditioner operator)
  // two-phase / transport fields (caller-owned nodal vectors) and the per-q coefficient
  // fields built from them (LAW 4 of the cell kernels), FP64 and its FP32 copy
  const double *Hf = nullptr, *vel = nullptr;
  double *cf = nullptr;
  float *cf_f = nullptr;
  bool cf_dirty = true, cf_f_dirty = true;
  // tangent coefficient fields of the LAW 5 operator at the linearisation point (8 per
  // point, for the register-resident kernel's LAW 6) and their FP32 copy
  double *tf = nullptr;
  float *tf_f = nullptr;
  bool tf_dirty = true, tf_f_dirty = true;
  // tangent fields of the linear-k law at the linearisation point (4 per point, LAW 7)
  double *tk = nullptr;
  bool tk_dirty = true;
  // GMRES basis (m + 1 vectors) and small device buffers
  double *gV = nullptr;
  int gV_m = 0;
  double *gsmall = nullptr;
  float *nn_buf = nullptr;  // learned guess: network input and output on the sampled grid
  // boundary terms per face: type bit 1 convection, 2 radiation, 4 Neumann
  int btype[6] = {0, 0, 0, 0, 0, 0};
  double bh[6] = {0}, bTc[6] = {0}, beps[6] = {0}, bTr[6] = {0}, bqn[6] = {0};
  double *face_dot = nullptr;
  int64_t nn_buf_n = 0;
  // reduction scratch
  double *partials = nullptr;
  unsigned *counter = nullptr;
  SolverState *st = nullptr, *st_host = nullptr;
  double *scal = nullptr, *scal_host = nullptr;
  // the page-locked st_host / scal_host / rd_host are mapped: st_map, scal_map and rd_map are
  // their device addresses, written by k_read_words (small reads then never wait behind a
  // bulk host copy on a copy engine)
  SolverState *st_map = nullptr;
  double *scal_map = nullptr, *rd_host = nullptr, *rd_map = nullptr;
  // Krylov / step workspace
  double *r = nullptr, *pv = nullptr, *Ap = nullptr, *z = nullptr, *w1 = nullptr, *w2 = nullptr,
         *w3 = nullptr;
  float *r32 = nullptr, *x32 = nullptr, *d32 = nullptr, *Ax32 = nullptr;
  // the fine level's Chebyshev iterate in the cell-row layout (instead of x32) during a mixed
  // solve whose preconditioner applies the FP32 Picard operator of FE_Q(3) (rows_on)
  float *x32_rows = nullptr;
  bool rows_on = false;
  double *host_T = nullptr, *host_To = nullptr, *host_q = nullptr;  // device buffers for *_host
  // host-vector verbs: device mirrors of the linearisation point and of the verb's vectors,
  // and the caller's DoF numbering (lex[i] = lexicographic index of the caller's DoF i)
  double *hv_T = nullptr, *hv_To = nullptr, *hv_a = nullptr, *hv_b = nullptr, *hv_c = nullptr;
  int64_t *perm = nullptr, *perm_buf = nullptr;  // perm: perm_buf while a permutation is set
  // mpdg_heat_set_laser: the residual evaluates this laser at the support points in place of a
  // NULL heat_source
  SourceEval source{};
  const double *guess = nullptr;
  // MPDG_PREDICTOR_LINEAR_DIRECTION: the increment direction d, and for the next solve the
  // operator applied to its initial guess (x_Ax_scale * x_Ax = A x, computed by the step)
  const double *direction = nullptr;
  const double *x_Ax = nullptr;
  double x_Ax_scale = 0.0;
  int64_t bytes = 0;
  std::vector<void *> owned;
  // instrumentation
  int64_t launches = 0, vm64 = 0, vm32 = 0;
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev64, ev32;
  std::vector<cudaEvent_t> ev_pool;
  double ms64 = 0.0, ms32 = 0.0;
  // p-multigrid preconditioner: levels and the scratch of the separable transfers
  std::vector<MGLevel> mg;
  float *mg_t1 = nullptr, *mg_t2 = nullptr;
  int mg_min_cells = -1;
  bool x_zero = false;  // the next solve starts from x = 0 (its A x is skipped)
  bool mixed_ready = false;  // mixed_prepare ran at the current linearisation point
  // host-buffer time step: a copy stream for the transfers that overlap the step, and the
  // events the step records / waits on (null outside mpdg_heat_time_step_host)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_source = nullptr, ev_commit = nullptr, ev_inputs = nullptr;
  bool wait_source = false, record_commit = false;
  double *told_host = nullptr;  // host destination of the committed T_old (copy stream)
  // resident host step: the new T = T_g + x formed in t_out as soon as the increment solve has
  // converged and sent to early_host on the copy stream, so that the download overlaps the FP64
  // residual recheck (early_T: the step's T_g; early_sent: that download holds the final T, no
  // restart changed the increment after it)
  double *early_host = nullptr, *early_T = nullptr, *t_out = nullptr;
  bool early_sent = false;
  cudaEvent_t ev_early = nullptr;
  // host-buffer steps: the source uploaded in n_slabs z-slabs of node planes (event ev_slab[k]
  // after slab k), so that create_rhs applies the cells of cell layers [slab_cz[k],
  // slab_cz[k + 1]) as soon as slab k has arrived (0: one upload, ev_source)
  static constexpr int kMaxSlabs = 4;
  int n_slabs = 0;
  int slab_cz[kMaxSlabs + 1] = {0};
  cudaEvent_t ev_slab[kMaxSlabs] = {};
  double *res_T = nullptr, *res_To = nullptr;  // device-resident history (time_step_resident)
  // the resident step swaps the roles of its two history buffers instead of copying T into
  // T_old (the predictor writes in place over T_{n-1}); rotated reports that the swap happened
  bool rotate = false, rotated = false;
  // one iteration of the mixed-precision CG as a CUDA graph (recorded on cap_stream, replayed
  // on stream) and the kernel launches / operator applications one replay performs
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t body_exec = nullptr;
  int64_t body_launches = 0, body_vm64 = 0, body_vm32 = 0;
  // flexible GMRES: the FP32 preconditioned directions (m vectors) and a solver state that
  // stays "running" for the Chebyshev kernels
  float *gZ = nullptr;
  int gZ_m = 0;
  SolverState *st_run = nullptr;
  // iterations of the last mixed-precision solve per preconditioner (0 multigrid, 1 Chebyshev):
  // the next solve issues that many before its first convergence poll
  int its_hint[2] = {0, 0};
  // FP32 Picard operator on the tensor cores (uniform box, FE_Q(3)): on/off (-1: the
  // MPDG_PICARD_TC setting, off unless it is 1), its G matrices (device, 2 x 64 KB), and a page-locked mapped flag the
  // kernel raises when a wait times out (tc_err_map: its device address)
  int picard_tc = -1;
  float *gmat_tc = nullptr;
  int *tc_err_host = nullptr, *tc_err_map = nullptr;
};

static cudaEvent_t take_event(mpdg_heat *h)
{
  if (!h->ev_pool.empty()) {
    cudaEvent_t e = h->ev_pool.back();
    h->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// fold recorded operator-timing events into the sums (stream must be idle)
static void drain_events(mpdg_heat *h)
{
  for (auto *v : {&h->ev64, &h->ev32}) {
    for (auto &pr : *v) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess)
        (v == &h->ev64 ? h->ms64 : h->ms32) += ms;
      h->ev_pool.push_back(pr.first);
      h->ev_pool.push_back(pr.second);
    }
    v->clear();
  }
}

static constexpr int kPartialsPerValue = 148 * 64;

static int dalloc(mpdg_heat *h, void **p, size_t bytes)
{
  if (*p) return MPDG_OK;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(MPDG_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  h->owned.push_back(*p);
  h->bytes += (int64_t)bytes;
  return MPDG_OK;
}
template <typename T> static int dvec(mpdg_heat *h, T **p, int64_t n)
{
  return dalloc(h, reinterpret_cast<void **>(p), sizeof(T) * (size_t)n);
}

// ---------------------------------------------------------------------------
// per-device table upload
// ---------------------------------------------------------------------------
static DegreeTable table_for(int n)
{
  switch (n) {
  case 2: return degree_table_2();
  case 3: return degree_table_3();
  case 4: return degree_table_4();
  case 5: return degree_table_5();
  case 6: return degree_table_6();
  default: return degree_table_7();
  }
}

static bool g_uploaded[64][8];

static int upload_tables(int device, int n)
{
  if (device < 0 || device >= 64) return fail(MPDG_ERR_INVALID_ARGUMENT, "device id");
  if (g_uploaded[device][n]) return MPDG_OK;
  std::vector<double> tab, w, xl;
  fill_even_odd(tab, w, xl);
  std::vector<float> tabf(tab.begin(), tab.end()), wf(w.begin(), w.end());
  table_for(n).upload(tab.data(), tabf.data(), w.data(), wf.data());
  CU(cudaGetLastError());
  g_uploaded[device][n] = true;
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------
// per-quadrature-point JxW and G = JxW J^-1 J^-T of the trilinear map
__global__ void k_geometry(int64_t n_cells, MeshDims d, int n, Q1D q1, const double *vert,
                           double *geo)
{
  const int npt = n * n * n;
  const int64_t total = n_cells * npt;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / npt;
    const int q = (int)(t % npt);
    const int qi = q % n, qj = (q / n) % n, qk = q / (n * n);
    const int cx = (int)(c % d.m[0]), cy = (int)((c / d.m[0]) % d.m[1]),
              cz = (int)(c / ((int64_t)d.m[0] * d.m[1]));
    const double xi[3] = {q1.xg[qi], q1.xg[qj], q1.xg[qk]};
    double x[3], J[3][3];
    trilinear(vert, d, cx, cy, cz, xi, x, J);
    const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                       J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                       J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    double inv[3][3];
    inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    const double w = q1.wg[qi] * q1.wg[qj] * q1.wg[qk];
    const double jxw = det * w;
    const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
    double *g = geo + c * 7 * npt + q;
    g[0] = jxw;
    for (int k = 0; k < 6; ++k) {
      double s = 0.0;
      for (int e = 0; e < 3; ++e) s += inv[ia[k]][e] * inv[ib[k]][e];
      g[(1 + k) * npt] = jxw * s;
    }
  }
}

// Per-quadrature-point coefficients of the gas-liquid / convective operator,
// cf[cell][5][npt] = {rho_cp JxW, k, JxW rho_cp J^-1 v} (mode 4; mode 5, for the laws that
// depend on T_lin, stores {w, 0, JxW J^-1 v} and the cell kernels evaluate the liquid-solid
// law and mix it with the gas by w): the heaviside and velocity fields
// are interpolated at the point (FEEvaluation::evaluate(values) on the nodal vectors,
// heat_diffuse_operator.cpp:448-473), the gas-liquid law mixes the phase properties with
// w = H (smooth) or w = (H > 0.5) (sharp): (1 - w) gas + w liquid
// (Material::compute_parameters, material.templates.hpp:240-295 and :515-524); rho_cp is
// the product of the mixed density and capacity or the mixed volume-specific capacity
// (heat_diffuse_operator.cpp:1138-1162).  Without a heaviside field w = 1 (liquid
// properties, the constant law).  J^-1 v turns v.grad(u) into a contraction with the
// reference gradient.  The field values at the points come from the sum-factorised
// k_field_values, written into the slots of cf that this kernel then overwrites (each thread
// reads and writes only its own point); one thread per (cell, point).
struct FieldArgs {
  MeshDims d;
  int n, geo, mode;
  int64_t n_cells, n_dofs;
  double hc[3];
  double xg[8], wg[8];
  const double *vert, *H, *vel;  // H, vel: presence flags (their values come through cf)
  int mix, sharp, vs;
  double rho_l, cp_l, k_l, rho_g, cp_g, k_g;
  double *cf;
};

__global__ void k_coef_fields(FieldArgs a)
{
  const int n = a.n, npt = n * n * n;
  const int64_t total = a.n_cells * npt;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / npt;
    const int q = (int)(t % npt);
    const int qi = q % n, qj = (q / n) % n, qk = q / (n * n);
    const int cx = (int)(c % a.d.m[0]), cy = (int)((c / a.d.m[0]) % a.d.m[1]),
              cz = (int)(c / ((int64_t)a.d.m[0] * a.d.m[1]));
    double *o = a.cf + c * 5 * npt + q;
    const double Hq = o[0];
    const double v[3] = {o[2 * npt], o[3 * npt], o[4 * npt]};
    const double w = !a.mix ? 1.0 : (!a.H ? 1.0 : (a.sharp ? (Hq > 0.5 ? 1.0 : 0.0) : Hq));
    const double kk = (1.0 - w) * a.k_g + w * a.k_l;
    const double rhocp = a.vs ? (1.0 - w) * (a.rho_g * a.cp_g) + w * (a.rho_l * a.cp_l)
                              : ((1.0 - w) * a.rho_g + w * a.rho_l) * ((1.0 - w) * a.cp_g + w * a.cp_l);
    double det, inv[3][3];
    if (a.geo == 0) {
      det = a.hc[0] * a.hc[1] * a.hc[2];
      for (int e = 0; e < 3; ++e)
        for (int f = 0; f < 3; ++f) inv[e][f] = e == f ? 1.0 / a.hc[e] : 0.0;
    } else {
      const double xi[3] = {a.xg[qi], a.xg[qj], a.xg[qk]};
      double x[3], J[3][3];
      trilinear(a.vert, a.d, cx, cy, cz, xi, x, J);
      det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
            J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
            J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
      for (int e = 0; e < 3; ++e)
        for (int f = 0; f < 3; ++f) {
          // (J^-1)[e][f] = cofactor of J[f][e] / det
          const int r0 = (f + 1) % 3, r1 = (f + 2) % 3, c0 = (e + 1) % 3, c1 = (e + 2) % 3;
          inv[e][f] = (J[r0][c0] * J[r1][c1] - J[r0][c1] * J[r1][c0]) / det;
        }
    }
    const double jxw = det * a.wg[qi] * a.wg[qj] * a.wg[qk];
    const double s = a.mode == 5 ? jxw : jxw * rhocp;
    o[0] = a.mode == 5 ? w : rhocp * jxw;
    o[npt] = a.mode == 5 ? 0.0 : kk;
    for (int e = 0; e < 3; ++e)
      o[(2 + e) * npt] = s * (inv[e][0] * v[0] + inv[e][1] * v[1] + inv[e][2] * v[2]);
  }
}

__global__ void k_support_points(int64_t N, PosArgs a, double *xyz)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N;
       i += (int64_t)gridDim.x * blockDim.x) {
    double x[3];
    dof_position(a, i, x);
    xyz[3 * i] = x[0];
    xyz[3 * i + 1] = x[1];
    xyz[3 * i + 2] = x[2];
  }
}

__global__ void k_gaussian(int64_t N, PosArgs a, double *q, double amp, double c0, double c1,
                           double c2, double inv_r2)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N;
       i += (int64_t)gridDim.x * blockDim.x) {
    double x[3];
    dof_position(a, i, x);
    const double d2 = (x[0] - c0) * (x[0] - c0) + (x[1] - c1) * (x[1] - c1) + (x[2] - c2) * (x[2] - c2);
    q[i] = amp * exp(-d2 * inv_r2);
  }
}

__global__ void k_laser(int64_t N, PosArgs a, LaserArgs g, double *q)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N;
       i += (int64_t)gridDim.x * blockDim.x) {
    double x[3];
    dof_position(a, i, x);
    q[i] = laser_intensity(g, x);
  }
}

// set Dirichlet values face by face; a DoF on several faces takes the value of
// the first constrained face in the order x-, x+, y-, y+, z-, z+
struct DirArgs {
  MeshDims d;
  double val[6];
};
__global__ void k_distribute(DirArgs a, int face, double *u)
{
  const int dir = face / 2;
  const int e1 = dir == 0 ? 1 : 0, e2 = dir == 2 ? 1 : 2;
  const int64_t n1 = a.d.nd[e1], n2 = a.d.nd[e2];
  const int fixed = (face & 1) ? a.d.nd[dir] - 1 : 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n1 * n2;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t pos[3];
    pos[dir] = fixed;
    pos[e1] = t % n1;
    pos[e2] = t / n1;
    bool earlier = false;
    for (int f = 0; f < face; ++f) {
      if (!(a.d.dmask & (1 << f))) continue;
      const int df = f / 2;
      const int64_t at = (f & 1) ? a.d.nd[df] - 1 : 0;
      if (pos[df] == at) earlier = true;
    }
    if (earlier) continue;
    const int64_t idx = pos[0] + (int64_t)a.d.nd[0] * (pos[1] + (int64_t)a.d.nd[1] * pos[2]);
    u[idx] = a.val[face];
  }
}

// ---------------------------------------------------------------------------
// vector kernels
// ---------------------------------------------------------------------------
#define GRID_STRIDE(i, N) \
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (N); i += (int64_t)gridDim.x * blockDim.x)

__global__ void k_cast_f(int64_t N, const double *__restrict__ x, float *__restrict__ y)
{
  GRID_STRIDE(i, N) y[i] = (float)x[i];
}
// inv = |d| > 1e-10 ? 1/d : 1 (the FP64 rule of compute_inverse_diagonal, in FP32)
__global__ void k_invert_diag_f(int64_t N, const float *__restrict__ d, float *inv)
{
  GRID_STRIDE(i, N)
  {
    const float v = d[i];
    inv[i] = fabsf(v) > 1.0e-10f ? 1.f / v : 1.f;
  }
}
__global__ void k_invert_diag(int64_t N, double *d)
{
  GRID_STRIDE(i, N)
  {
    const double v = d[i];
    d[i] = fabs(v) > 1.0e-10 ? 1.0 / v : 1.0;
  }
}
__global__ void k_scale(int64_t N, double *dst, const double *__restrict__ src,
                        const double *__restrict__ D)
{
  GRID_STRIDE(i, N) dst[i] = src[i] * D[i];
}
__global__ void k_predict(int64_t N, const double *__restrict__ T, const double *__restrict__ To,
                          double *out, double f)
{
  GRID_STRIDE(i, N) out[i] = (f + 1.0) * T[i] - f * To[i];
}
// the same extrapolation written over T_{n-1} (each entry is read before it is written)
__global__ void k_predict_inplace(int64_t N, const double *__restrict__ T, double *To, double f)
{
  GRID_STRIDE(i, N) To[i] = (f + 1.0) * T[i] - f * To[i];
}
__global__ void k_axpy(int64_t N, double *y, double a, const double *__restrict__ x)
{
  GRID_STRIDE(i, N) y[i] += a * x[i];
}
// out = a + b (the same sum k_axpy forms with a = 1)
__global__ void k_sum(int64_t N, double *out, const double *__restrict__ a,
                      const double *__restrict__ b)
{
  GRID_STRIDE(i, N) out[i] = a[i] + b[i];
}
__global__ void k_masked_random(int64_t N, MeshDims d, double *b)
{
  GRID_STRIDE(i, N)
  {
    const int64_t I = i % d.nd[0], J = (i / d.nd[0]) % d.nd[1], K = i / ((int64_t)d.nd[0] * d.nd[1]);
    uint64_t x = 0x9E3779B97F4A7C15ULL * (uint64_t)(i + 1) + 0x632BE59BD9B4E019ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    x ^= x >> 31;
    const bool c = ((d.dmask & 1) && I == 0) || ((d.dmask & 2) && I == d.nd[0] - 1) ||
                   ((d.dmask & 4) && J == 0) || ((d.dmask & 8) && J == d.nd[1] - 1) ||
                   ((d.dmask & 16) && K == 0) || ((d.dmask & 32) && K == d.nd[2] - 1);
    b[i] = c ? 0.0 : 2.0 * ((double)(x >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
  }
}

// sums[0] = a.a, sums[1] = (a+b).(a+b) (b may be null), written to out[0..1]
__global__ void k_norms(int64_t N, const double *__restrict__ a, const double *__restrict__ b,
                        double *partials, unsigned *counter, double *out)
{
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(i, N)
  {
    const double x = a[i];
    v[0] += x * x;
    const double y = b ? x + b[i] : x;
    v[1] += y * y;
  }
  double tot[2];
  if (grid_sum<2>(v, partials, counter, tot)) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

// ---- Jacobi / identity preconditioned CG (FP64) ----------------------------
// init: r = b - Ax ; z = D r ; p = z ; Ap = 0 ; rz, rr -> state
__global__ void k_cg_init(int64_t N, const double *__restrict__ b, double *r, double *p,
                          double *Ap, const double *__restrict__ D, SolverState *st,
                          double *partials, unsigned *counter, double rel, double abs_tol,
                          double ref_norm, int max_it, int record)
{
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(i, N)
  {
    const double ri = b[i] - Ap[i];
    const double zi = D ? D[i] * ri : ri;
    r[i] = ri;
    p[i] = zi;
    Ap[i] = 0.0;
    v[0] += ri * zi;
    v[1] += ri * ri;
  }
  double tot[2];
  if (grid_sum<2>(v, partials, counter, tot)) {
    st->rz = tot[0];
    st->rr = tot[1];
    st->res = st->res0 = sqrt(tot[1]);
    st->tol = fmax(abs_tol, rel * (ref_norm > 0.0 ? ref_norm : st->res0));
    st->it = 0;
    st->max_it = max_it;
    st->status = 0;
    st->first = 1;
    st->record = record;
    st->alpha = st->beta = 0.0;
    if (!isfinite(st->res)) {
      st->done = 2;
      st->status = MPDG_ERR_NAN;
    } else if (st->res <= st->tol) {
      st->done = 1;
    } else if (max_it <= 0) {
      st->done = 2;
      st->status = MPDG_ERR_NOT_CONVERGED;
    } else {
      st->done = 0;
    }
  }
}

__device__ __forceinline__ void finish_iteration(SolverState *st, double rr)
{
  const int it = ++st->it;
  st->rr = rr;
  st->res = sqrt(rr);
  if (st->record && it <= 64) {
    st->hist_alpha[it - 1] = st->alpha;
    st->hist_beta[it - 1] = st->beta;
  }
  if (!isfinite(st->res)) {
    st->done = 2;
    st->status = MPDG_ERR_NAN;
  } else if (st->res <= st->tol) {
    st->done = 1;
  } else if (it >= st->max_it) {
    st->done = 2;
    st->status = MPDG_ERR_NOT_CONVERGED;
  }
}

// x += alpha p ; r -= alpha Ap ; rz = r.D r ; rr = r.r ; beta = rz / rz_old
__global__ void k_cg_update_xr(int64_t N, double *x, double *r, const double *__restrict__ p,
                               const double *__restrict__ Ap, const double *__restrict__ D,
                               SolverState *st, double *partials, unsigned *counter)
{
  if (st->done) return;
  const double alpha = st->alpha;
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(i, N)
  {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    const double zi = D ? D[i] * ri : ri;
    v[0] += ri * zi;
    v[1] += ri * ri;
  }
  double tot[2];
  if (grid_sum<2>(v, partials, counter, tot)) {
    st->beta = tot[0] / st->rz;
    st->rz_old = st->rz;
    st->rz = tot[0];
    finish_iteration(st, tot[1]);
  }
}

// p = D r + beta p ; Ap = 0
__global__ void k_cg_update_p(int64_t N, const double *__restrict__ r, double *p, double *Ap,
                              const double *__restrict__ D, const SolverState *st)
{
  if (st->done) return;
  const double beta = st->beta;
  GRID_STRIDE(i, N)
  {
    const double zi = D ? D[i] * r[i] : r[i];
    p[i] = zi + beta * p[i];
    Ap[i] = 0.0;
  }
}

// ---- the cell-row layout of the fine level's FP32 iterate -------------------
// FE_Q(3): x-row r of the nodal grid (r = j + nd1 k) holds 4 slots per cell column c, slot s
// holding node 3c + s, so that a cell's 4 x-nodes are one aligned float4 (the operator's
// gather, k_vmult2 with ROWS); node 3c, shared by columns c - 1 and c, is in both (slot 3 of
// c - 1 and slot 0 of c). rows == nullptr: the iterate is the lexicographic x32. Node indices
// are below 2^32 (checked where the layout is enabled).
struct CellRows {
  float *rows = nullptr;
  unsigned nd0 = 0;  // nodes per x-row, 3 m0 + 1
  unsigned rs = 0;   // slots per x-row, 4 m0
};

__device__ __forceinline__ float *cell_row_of(const CellRows &c, int64_t i, unsigned &ix)
{
  const unsigned ii = (unsigned)i, r = ii / c.nd0;
  ix = ii - r * c.nd0;
  return c.rows + (int64_t)r * c.rs;
}
// x[i] into every slot of node i
__device__ __forceinline__ void cell_rows_store(const CellRows &c, int64_t i, float v)
{
  unsigned ix;
  float *row = cell_row_of(c, i, ix);
  const unsigned q = ix / 3u, s = ix - 3u * q;
  if (ix + 1u < c.nd0) row[ix + q] = v;  // slot s of column q (the row's last node has none)
  if (s == 0u && q > 0u) row[ix + q - 1u] = v;  // slot 3 of column q - 1
}
__device__ __forceinline__ float cell_rows_load(const CellRows &c, int64_t i)
{
  unsigned ix;
  const float *row = cell_row_of(c, i, ix);
  const unsigned q = ix / 3u;
  return row[ix + 1u < c.nd0 ? ix + q : ix + q - 1u];
}

// the handle's fine-level iterate: its cell rows while rows_on, else the lexicographic x32
static CellRows cell_rows_of(const mpdg_heat *h)
{
  CellRows c;
  if (h->rows_on) {
    c.rows = h->x32_rows;
    c.nd0 = (unsigned)h->dims.nd[0];
    c.rs = 4u * (unsigned)h->dims.m[0];
  }
  return c;
}
static int64_t cell_rows_size(const mpdg_heat *h)
{
  return (int64_t)4 * h->dims.m[0] * h->dims.nd[1] * h->dims.nd[2];
}

// ---- FP64 CG with the FP32 Chebyshev-Jacobi preconditioner ------------------
// init: r = b - Ax ; rr ; r32 = r ; x32 = D32 r32 / theta ; d32 = x32 ; Ap = 0 ; Ax32 = 0
// (x32 into xr's cell rows instead with ROWS)
template <bool ROWS>
__global__ void k_cgm_init(int64_t N, const double *__restrict__ b, double *r, double *Ap,
                           float *r32, float *x32, float *d32, float *Ax32,
                           const float *__restrict__ D32, float inv_theta, SolverState *st,
                           double *partials, unsigned *counter, double rel, double abs_tol,
                           double ref_norm, int max_it, CellRows xr)
{
  double v[1] = {0.0};
  GRID_STRIDE(i, N)
  {
    const double ri = b[i] - Ap[i];
    r[i] = ri;
    Ap[i] = 0.0;
    const float rf = (float)ri;
    r32[i] = rf;
    const float xf = D32[i] * rf * inv_theta;
    if constexpr (ROWS)
      cell_rows_store(xr, i, xf);
    else
      x32[i] = xf;
    d32[i] = xf;
    Ax32[i] = 0.0f;
    v[0] += ri * ri;
  }
  double tot[1];
  if (grid_sum<1>(v, partials, counter, tot)) {
    st->rr = tot[0];
    st->res = st->res0 = sqrt(tot[0]);
    st->tol = fmax(abs_tol, rel * (ref_norm > 0.0 ? ref_norm : st->res0));
    st->it = 0;
    st->max_it = max_it;
    st->status = 0;
    st->first = 1;
    st->record = 0;
    st->alpha = st->beta = 0.0;
    if (!isfinite(st->res)) {
      st->done = 2;
      st->status = MPDG_ERR_NAN;
    } else if (st->res <= st->tol) {
      st->done = 1;
    } else if (max_it <= 0) {
      st->done = 2;
      st->status = MPDG_ERR_NOT_CONVERGED;
    } else {
      st->done = 0;
    }
  }
}

// Chebyshev step: d = c1 d + c2 D32 (r32 - Ax32) ; x32 += d ; Ax32 = 0
// (x in xr's cell rows instead of x32 with ROWS)
template <bool ROWS>
__global__ void k_cheb_step(int64_t N, const float *__restrict__ r32, float *x32, float *d32,
                            float *Ax32, const float *__restrict__ D32, float c1, float c2,
                            const SolverState *st, CellRows xr)
{
  if (st->done) return;
  GRID_STRIDE(i, N)
  {
    const float dn = c1 * d32[i] + c2 * D32[i] * (r32[i] - Ax32[i]);
    d32[i] = dn;
    if constexpr (ROWS)
      cell_rows_store(xr, i, cell_rows_load(xr, i) + dn);
    else
      x32[i] += dn;
    Ax32[i] = 0.0f;
  }
}

// last Chebyshev step, then z = x32 (FP64), rz = r.z, zAp = z.Ap and the
// flexible (Polak-Ribiere) beta = z.(r - r_old) / rz_old = -alpha z.Ap / rz_old
// (x in xr's cell rows instead of x32 with ROWS)
template <bool ROWS>
__global__ void k_cheb_last(int64_t N, const float *__restrict__ r32, const float *__restrict__ x32,
                            const float *__restrict__ d32, float *Ax32,
                            const float *__restrict__ D32, float c1, float c2,
                            const double *__restrict__ r, const double *__restrict__ Ap, double *z,
                            SolverState *st, double *partials, unsigned *counter, CellRows xr)
{
  if (st->done) return;
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(i, N)
  {
    const float dn = c1 * d32[i] + c2 * D32[i] * (r32[i] - Ax32[i]);
    float xi;
    if constexpr (ROWS)
      xi = cell_rows_load(xr, i);
    else
      xi = x32[i];
    const double zi = (double)(xi + dn);
    Ax32[i] = 0.0f;
    z[i] = zi;
    v[0] += zi * r[i];
    v[1] += zi * Ap[i];
  }
  double tot[2];
  if (grid_sum<2>(v, partials, counter, tot)) {
    if (st->first) {
      st->beta = 0.0;
      st->first = 0;
    } else {
      st->beta = -st->alpha * tot[1] / st->rz;
    }
    st->rz = tot[0];
    st->zAp = tot[1];
  }
}

// x += alpha p ; r -= alpha Ap ; rr ; r32 = r ; x32 = D32 r32 / theta ; d32 = x32
template <bool ROWS>
__global__ void k_cgm_update_xr(int64_t N, double *x, double *r, const double *__restrict__ p,
                                const double *__restrict__ Ap, float *r32, float *x32, float *d32,
                                const float *__restrict__ D32, float inv_theta, SolverState *st,
                                double *partials, unsigned *counter, CellRows xr)
{
  if (st->done) return;
  const double alpha = st->alpha;
  double v[1] = {0.0};
  GRID_STRIDE(i, N)
  {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    const float rf = (float)ri;
    r32[i] = rf;
    const float xf = D32[i] * rf * inv_theta;
    if constexpr (ROWS)
      cell_rows_store(xr, i, xf);
    else
      x32[i] = xf;
    d32[i] = xf;
    v[0] += ri * ri;
  }
  double tot[1];
  if (grid_sum<1>(v, partials, counter, tot)) finish_iteration(st, tot[0]);
}

// p = z + beta p ; Ap = 0
__global__ void k_cgm_update_p(int64_t N, const double *__restrict__ z, double *p, double *Ap,
                               const SolverState *st)
{
  if (st->done) return;
  const double beta = st->beta;
  GRID_STRIDE(i, N)
  {
    p[i] = beta != 0.0 ? z[i] + beta * p[i] : z[i];  // first direction: p = z
    Ap[i] = 0.0;
  }
}

// ---- p-multigrid building blocks ---------------------------------------------
struct Dims3 {
  int n[3];
  __host__ __device__ int64_t size() const { return (int64_t)n[0] * n[1] * n[2]; }
  __host__ __device__ int64_t at(int i, int j, int k) const
  {
    return i + (int64_t)n[0] * (j + (int64_t)n[1] * k);
  }
};
struct Transfer1D {
  int r;         // fine nodes per coarse interval
  float xi[8];   // position of fine node a (0 <= a < r) in its coarse interval
};

// coarse[V] = fine[r V] per direction (FP64 linearisation point)
__global__ void k_inject(Dims3 fd, Dims3 cd, int r, const double *__restrict__ fine,
                         double *coarse)
{
  GRID_STRIDE(i, cd.size())
  {
    const int a = (int)(i % cd.n[0]), b = (int)((i / cd.n[0]) % cd.n[1]),
              c = (int)(i / ((int64_t)cd.n[0] * cd.n[1]));
    coarse[i] = fine[fd.at(r * a, r * b, r * c)];
  }
}

// The transfer kernels index with 32 bits (every level holds < 2^31 nodes): a
// grid-stride loop over the flattened output with unsigned 32-bit div/mod.
#define TRANSFER_LOOP(i, d)                                                                  \
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < (unsigned)(d).size();       \
       i += gridDim.x * blockDim.x)
__device__ __forceinline__ void transfer_index(const Dims3 &d, unsigned i, int o[3])
{
  const unsigned r = i / (unsigned)d.n[0];
  o[0] = (int)(i - r * (unsigned)d.n[0]);
  o[2] = (int)(r / (unsigned)d.n[1]);
  o[1] = (int)(r - (unsigned)o[2] * (unsigned)d.n[1]);
}

// restriction along one axis (transpose of the interpolation below):
// out[.., V, ..] = sum_{|s| < r} phi_V(node r V + s) in[.., r V + s, ..]; with sub, the
// input is b - in (the residual of the smoothed iterate, formed on the fly); masked rows
// of the coarse level are set to zero
__global__ void k_restrict_axis(int axis, Dims3 di, Dims3 dout, Transfer1D t,
                                const float *__restrict__ in, const float *__restrict__ sub_b,
                                float *out, MeshDims md, int masked, const SolverState *st)
{
  if (st && st->done) return;
  TRANSFER_LOOP(i, dout)
  {
    int o[3];
    transfer_index(dout, i, o);
    if (masked && constrained(md, o[0], o[1], o[2])) {
      out[i] = 0.f;
      continue;
    }
    const int V = o[axis];
    float acc = 0.f;
    for (int s = -(t.r - 1); s <= t.r - 1; ++s) {
      const int I = t.r * V + s;
      if (I < 0 || I >= di.n[axis]) continue;
      const float w = s == 0 ? 1.f : (s > 0 ? 1.f - t.xi[s] : t.xi[t.r + s]);
      int p[3] = {o[0], o[1], o[2]};
      p[axis] = I;
      const unsigned j = (unsigned)p[0] + (unsigned)di.n[0] * ((unsigned)p[1] + (unsigned)di.n[1] * (unsigned)p[2]);
      acc += w * (sub_b ? sub_b[j] - in[j] : in[j]);
    }
    out[i] = acc;
  }
}

// interpolation along one axis: out[.., I, ..] = (1 - xi_a) in[.., V, ..] + xi_a in[.., V + 1, ..]
// with V = I / r, a = I % r; add: accumulate into out; masked rows are left untouched;
// zero (optional): an array of out's shape set to zero on the way; out in xr's cell rows
// instead with ROWS
template <bool ROWS>
__global__ void k_prolong_axis(int axis, Dims3 di, Dims3 dout, Transfer1D t,
                               const float *__restrict__ in, float *out, int add, MeshDims md,
                               int masked, float *zero, const SolverState *st, CellRows xr)
{
  if (st && st->done) return;
  TRANSFER_LOOP(i, dout)
  {
    int o[3];
    transfer_index(dout, i, o);
    if (zero) zero[i] = 0.f;
    if (masked && constrained(md, o[0], o[1], o[2])) {
      if (!add) {
        if constexpr (ROWS)
          cell_rows_store(xr, i, 0.f);
        else
          out[i] = 0.f;
      }
      continue;
    }
    const int I = o[axis], V = I / t.r, a = I - V * t.r;
    int p[3] = {o[0], o[1], o[2]};
    p[axis] = V;
    float v = in[(unsigned)p[0] + (unsigned)di.n[0] * ((unsigned)p[1] + (unsigned)di.n[1] * (unsigned)p[2])];
    if (a != 0) {
      p[axis] = V + 1;
      v = (1.f - t.xi[a]) * v +
          t.xi[a] * in[(unsigned)p[0] + (unsigned)di.n[0] * ((unsigned)p[1] + (unsigned)di.n[1] * (unsigned)p[2])];
    }
    if constexpr (ROWS)
      cell_rows_store(xr, i, add ? cell_rows_load(xr, i) + v : v);
    else
      out[i] = add ? out[i] + v : v;
  }
}

// first Chebyshev step from zero: x = d = D b / theta
__global__ void k_cheb_init(int64_t N, const float *__restrict__ b, float *x, float *d,
                            const float *__restrict__ D32, float inv_theta, const SolverState *st)
{
  if (st->done) return;
  GRID_STRIDE(i, N)
  {
    const float v = D32[i] * b[i] * inv_theta;
    x[i] = v;
    d[i] = v;
  }
}


// ---- GMRES building blocks --------------------------------------------------
constexpr int kMaxBasis = 32;

// out[i] = V_i . w for i < nv (V_i = V + i * ld)
// A CTA stages a chunk of w (kDotChunk values) in shared memory, then streams each V_i over
// the chunk (coalesced), each warp accumulating into its own shared slot per vector (fixed
// summation order: deterministic); the last CTA sums the nv per-CTA totals. Every vector and
// w are read once from memory, and the work per element is one load and one FMA whatever nv
// is (launch with VT = 256 threads).
constexpr int kDotChunk = 2048;
__global__ void __launch_bounds__(256) k_multidot(int64_t N, const double *__restrict__ V,
                                                  int64_t ld, int nv,
                                                  const double *__restrict__ w,
                                                  double *partials, unsigned *counter,
                                                  double *out)
{
  __shared__ double ws[kDotChunk];
  __shared__ double acc[kMaxBasis][8];  // [vector][warp]
  __shared__ int is_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int t = threadIdx.x; t < kMaxBasis * 8; t += blockDim.x) acc[t / 8][t % 8] = 0.0;
  for (int64_t c0 = (int64_t)blockIdx.x * kDotChunk; c0 < N;
       c0 += (int64_t)gridDim.x * kDotChunk) {
    const int len = (int)min((int64_t)kDotChunk, N - c0);
    __syncthreads();  // previous chunk's readers are done with ws
    for (int t = threadIdx.x; t < len; t += blockDim.x) ws[t] = w[c0 + t];
    __syncthreads();
    for (int i = 0; i < nv; ++i) {
      const double *vi = V + (int64_t)i * ld + c0;
      double s = 0.0;
      for (int t = threadIdx.x; t < len; t += blockDim.x) s += ws[t] * vi[t];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) acc[i][warp] += s;
    }
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double s = 0.0;
    for (int q = 0; q < nwarp; ++q) s += acc[threadIdx.x][q];
    partials[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  for (int i = warp; i < nv; i += nwarp) {
    double s = 0.0;
    for (unsigned b = lane; b < gridDim.x; b += 32) s += __ldcg(partials + (size_t)i * gridDim.x + b);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[i] = s;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// w -= sum_i c_i V_i (i < nv)
__global__ void k_multi_axpy(int64_t N, const double *__restrict__ V, int64_t ld, int nv,
                             const double *__restrict__ c, double *w)
{
  GRID_STRIDE(k, N)
  {
    double s = w[k];
    for (int i = 0; i < nv; ++i) s -= c[i] * V[(int64_t)i * ld + k];
    w[k] = s;
  }
}

// v = v * a ; z = D v (or v)
__global__ void k_scale_precond(int64_t N, double *v, double a, const double *__restrict__ D,
                                double *z)
{
  GRID_STRIDE(k, N)
  {
    const double x = v[k] * a;
    v[k] = x;
    z[k] = D ? D[k] * x : x;
  }
}

// v = b - Ax
__global__ void k_residual(int64_t N, const double *__restrict__ b, const double *__restrict__ Ax,
                           double *v)
{
  GRID_STRIDE(k, N) v[k] = b[k] - Ax[k];
}

// x += D (sum_i y_i V_i)
__global__ void k_gmres_update(int64_t N, const double *__restrict__ V, int64_t ld, int nv,
                               const double *__restrict__ y, const double *__restrict__ D,
                               double *x)
{
  GRID_STRIDE(k, N)
  {
    double s = 0.0;
    for (int i = 0; i < nv; ++i) s += y[i] * V[(int64_t)i * ld + k];
    x[k] += D ? D[k] * s : s;
  }
}

// ---- flexible GMRES with the FP32 Chebyshev-Jacobi preconditioner -----------
// Chebyshev start from the FP64 direction v: r32 = v ; x32 = D32 r32 / theta ; d32 = x32
__global__ void k_fgm_cheb_start(int64_t N, const double *__restrict__ v, float *r32, float *x32,
                                 float *d32, float *Ax32, const float *__restrict__ D32,
                                 float inv_theta)
{
  GRID_STRIDE(k, N)
  {
    const float rf = (float)v[k];
    r32[k] = rf;
    const float xf = D32[k] * rf * inv_theta;
    x32[k] = xf;
    d32[k] = xf;
    Ax32[k] = 0.0f;
  }
}

// z = x32 widened to FP64 (exact)
__global__ void k_widen(int64_t N, const float *__restrict__ x32, double *z)
{
  GRID_STRIDE(k, N) z[k] = (double)x32[k];
}

// x += sum_i y_i Z_i with the FP32-stored preconditioned directions Z_i (widened exactly)
__global__ void k_fgmres_update(int64_t N, const float *__restrict__ Z, int64_t ld, int nv,
                                const double *__restrict__ y, double *x)
{
  GRID_STRIDE(k, N)
  {
    double s = 0.0;
    for (int i = 0; i < nv; ++i) s += y[i] * (double)Z[(int64_t)i * ld + k];
    x[k] += s;
  }
}

// ---- boundary faces (Robin / Neumann) ----------------------------------------
// heat_diffuse_operator.cpp:243-269 (tangent loop), :719-781 (rhs loop),
// :1088-1129 (local face operation). Boundary vertices are never perturbed, so
// every boundary face is a flat h_a x h_b rectangle with JxW = h_a h_b w_a w_b.
constexpr double kStefanBoltzmann = 5.670374419e-8;  // physical_constants.hpp:6

template <typename T>
struct FaceArgs {
  MeshDims d;
  int n, face, dir, ea, eb, fixed, type;
  T ha, hb, hconv, Tinf_c, eps_sigma, Tinf_r4, qn;
  T S[kMaxN][kMaxN], w[kMaxN];
  const T *src;
  T *dst;
  const T *Tl;
  double *dot;          // += sum over faces of src.dst (vmult), nullable
  const SolverState *st;
};

// op 0: tangent (dst += A_f src), 1: rhs (dst += -R_f(Tl)), 2: diagonal
template <typename T, int OP>
__global__ void k_face(FaceArgs<T> a)
{
  if (a.st && a.st->done) return;
  __shared__ T s_u[kMaxN * kMaxN], s_T[kMaxN * kMaxN], s_v[kMaxN * kMaxN];
  __shared__ double s_red[32];
  const int n = a.n, nn = n * n;
  const int ca = blockIdx.x % a.d.m[a.ea], cb = blockIdx.x / a.d.m[a.ea];
  const int tid = threadIdx.x;
  const int ia = tid % n, ib = tid / n;
  int64_t g = 0;
  bool c = true;
  if (tid < nn) {
    int64_t pos[3];
    pos[a.dir] = a.fixed;
    pos[a.ea] = (int64_t)a.d.p * ca + ia;
    pos[a.eb] = (int64_t)a.d.p * cb + ib;
    g = pos[0] + (int64_t)a.d.nd[0] * (pos[1] + (int64_t)a.d.nd[1] * pos[2]);
    c = constrained(a.d, (int)pos[0], (int)pos[1], (int)pos[2]);
    s_u[tid] = (OP == 0 && !c) ? a.src[g] : T(0);
    s_T[tid] = a.Tl ? a.Tl[g] : T(0);
  }
  __syncthreads();
  if (tid < nn) {  // thread = quadrature point (qa, qb) = (ia, ib)
    T uq = 0, Tq = 0;
    for (int jb = 0; jb < n; ++jb)
      for (int ja = 0; ja < n; ++ja) {
        const T ph = a.S[ia][ja] * a.S[ib][jb];
        uq += ph * s_u[ja + n * jb];
        Tq += ph * s_T[ja + n * jb];
      }
    const T jxw = a.ha * a.hb * a.w[ia] * a.w[ib];
    T val = 0;
    if (OP == 1) {
      if (a.type & 4) val -= a.qn;
      if (a.type & 2) val -= a.eps_sigma * (Tq * Tq * Tq * Tq - a.Tinf_r4);
      if (a.type & 1) val -= a.hconv * (Tq - a.Tinf_c);
    } else {
      if (a.type & 1) val += a.hconv;
      if (a.type & 2) val += T(4) * a.eps_sigma * Tq * Tq * Tq;
      if (OP == 0) val *= uq;
    }
    s_v[tid] = val * jxw;
  }
  __syncthreads();
  double dot = 0.0;
  if (tid < nn) {  // thread = face DoF (ia, ib)
    T r = 0;
    for (int qb = 0; qb < n; ++qb)
      for (int qa = 0; qa < n; ++qa) {
        const T ph = a.S[qa][ia] * a.S[qb][ib];
        r += (OP == 2 ? ph * ph : ph) * s_v[qa + n * qb];
      }
    if (!c) {
      atomicAdd(a.dst + g, r);
      if (OP == 0) dot = (double)s_u[tid] * (double)r;
    }
  }
  if (OP == 0 && a.dot) {
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, o);
    if ((tid & 31) == 0) s_red[tid >> 5] = dot;
    __syncthreads();
    if (tid == 0) {
      double sacc = 0.0;
      for (int i = 0; i < (int)((blockDim.x + 31) >> 5); ++i) sacc += s_red[i];
      atomicAdd(a.dot, sacc);
    }
  }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
static int vgrid(const mpdg_heat *h, int64_t N)
{
  int64_t g = (N + VT - 1) / VT;
  const int64_t cap = (int64_t)h->sm_count * 8;
  if (g > cap) g = cap;
  return (int)std::max<int64_t>(g, 1);
}

__global__ void k_zero16(int64_t n, uint4 *p)
{
  GRID_STRIDE(i, n) p[i] = make_uint4(0u, 0u, 0u, 0u);
}
__global__ void k_zero4(int64_t n, unsigned *p)
{
  GRID_STRIDE(i, n) p[i] = 0u;
}

// zero fill by a kernel: a cudaMemsetAsync is not a kernel launch and can queue on a copy
// engine behind a bulk host copy in flight on another stream (the host step's T_old download)
static cudaError_t zero_async(mpdg_heat *h, void *p, size_t bytes, cudaStream_t s)
{
  if (bytes == 0) return cudaSuccess;
  const uintptr_t a = reinterpret_cast<uintptr_t>(p) | (uintptr_t)bytes;
  if (a % 16 == 0) {
    const int64_t n = (int64_t)(bytes / 16);
    k_zero16<<<vgrid(h, n), VT, 0, s>>>(n, static_cast<uint4 *>(p));
  } else if (a % 4 == 0) {
    const int64_t n = (int64_t)(bytes / 4);
    k_zero4<<<vgrid(h, n), VT, 0, s>>>(n, static_cast<unsigned *>(p));
  } else {
    return cudaMemsetAsync(p, 0, bytes, s);
  }
  ++h->launches;
  return cudaGetLastError();
}

template <typename T>
static CellArgs<T> cell_args(mpdg_heat *h)
{
  CellArgs<T> a;
  memset(&a, 0, sizeof(a));
  a.n_cells = h->n_cells;
  a.d = h->dims;
  const double detJ = h->hcell[0] * h->hcell[1] * h->hcell[2];
  a.g.detJ = (T)detJ;
  for (int e = 0; e < 3; ++e) a.g.Gd[e] = (T)(detJ / (h->hcell[e] * h->hcell[e]));
  a.g.q = nullptr;
  const mpdg_material &m = h->mat;
  a.m.rho_l = (T)m.rho_l;
  a.m.cp_l = (T)m.cp_l;
  a.m.k_l = (T)m.k_l;
  a.m.rho_s = (T)m.rho_s;
  a.m.cp_s = (T)m.cp_s;
  a.m.k_s = (T)m.k_s;
  a.m.rho_g = (T)m.rho_g;
  a.m.cp_g = (T)m.cp_g;
  a.m.k_g = (T)m.k_g;
  a.m.T_liq = (T)m.T_liquidus;
  a.m.T_sol = (T)m.T_solidus;
  a.m.inv_mushy = (T)(m.T_liquidus != m.T_solidus ? 1.0 / (m.T_liquidus - m.T_solidus) : 0.0);
  a.m.k1 = (T)m.k1;
  a.m.idt = (T)(1.0 / h->dt);
  a.m.sharp = m.sharp;
  a.m.vs = m.volume_specific;
  a.m.need_told = h->need_told;
  a.m.latent = (T)h->latent;
  a.m.acap = h->acap;
  a.partials = h->partials;
  a.counter = h->counter;
  a.fin = FIN_NONE;
  return a;
}

static int ensure_dt(mpdg_heat *h)
{
  if (!(h->dt != 0.0) || !std::isfinite(h->dt))
    return fail(MPDG_ERR_ZERO_TIME_INCREMENT, "time increment is zero: call reset_time_increment");
  return MPDG_OK;
}

// the cell kernels' law: the public laws 0-2; 4 (coefficient fields) for the gas-liquid law
// and the constant law with a velocity; 5 (liquid-solid law at T_lin mixed with the gas by a
// per-point weight, convection included) for the three-phase law and the liquid-solid law
// with a velocity (a velocity with the linear-k law is rejected)
static int klaw(const mpdg_heat *h)
{
  if (h->law == MPDG_LAW_GAS_LIQUID_SOLID || (h->law == MPDG_LAW_LIQUID_SOLID && h->vel)) return 5;
  if (h->law == MPDG_LAW_GAS_LIQUID || h->vel) return 4;
  return h->law;
}

static bool law_tdep(const mpdg_heat *h)
{
  return h->law == MPDG_LAW_LINEAR_K || h->law == MPDG_LAW_LIQUID_SOLID ||
         h->law == MPDG_LAW_GAS_LIQUID_SOLID;
}

// (re)build the per-q coefficient fields when the operator uses them
static int ensure_fields(mpdg_heat *h)
{
  if (klaw(h) < 4 || !h->cf_dirty) return MPDG_OK;
  TRY(dvec(h, &h->cf, h->n_cells * 5 * h->npt));
  const Tables1D t1 = make_tables(h->n);
  FieldArgs a;
  memset(&a, 0, sizeof(a));
  a.d = h->dims;
  a.n = h->n;
  a.geo = h->geo;
  a.mode = klaw(h);
  a.n_cells = h->n_cells;
  a.n_dofs = h->n_dofs;
  for (int e = 0; e < 3; ++e) a.hc[e] = h->hcell[e];
  for (int q = 0; q < h->n; ++q) {
    a.xg[q] = t1.xg[q];
    a.wg[q] = t1.wg[q];
  }
  a.vert = h->vert;
  a.H = h->Hf;
  a.vel = h->vel;
  a.mix = h->law == MPDG_LAW_GAS_LIQUID || h->law == MPDG_LAW_GAS_LIQUID_SOLID;
  a.sharp = h->mat.sharp_gas_liquid;
  a.vs = h->mat.volume_specific;
  a.rho_l = h->mat.rho_l;
  a.cp_l = h->mat.cp_l;
  a.k_l = h->mat.k_l;
  a.rho_g = h->mat.rho_g;
  a.cp_g = h->mat.cp_g;
  a.k_g = h->mat.k_g;
  a.cf = h->cf;
  {
    CellArgs<double> ca = cell_args<double>(h);
    CU(h->tab.field_values(ca, h->Hf, h->vel, h->n_dofs, h->cf, h->stream, h->sm_count));
    ++h->launches;
  }
  const int64_t total = h->n_cells * h->npt;
  k_coef_fields<<<vgrid(h, total), VT, 0, h->stream>>>(a); ++h->launches;
  CU(cudaGetLastError());
  h->cf_dirty = false;
  h->cf_f_dirty = true;
  return MPDG_OK;
}

// The linear-k tangent from fields built once per linearisation (LAW 7) instead of
// re-evaluating T_lin in every application; MPDG_TANGENT_FIELDS=0 keeps the evaluation.
static bool tangent_fields_enabled()
{
  static const int on = [] {
    const char *e = getenv("MPDG_TANGENT_FIELDS");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return on != 0;
}

// line-per-thread kernel (FP64, p >= 4) on deformed meshes: the linear-k tangent from the
// fields (preloaded with the geometry) instead of evaluating T_lin. The default at p = 4 and 6,
// where it measured faster per application (3.84 -> 3.26 ms and 4.64 -> 4.00 ms at ~57 M DoFs)
// and per production step with the fields' build included; at p = 5 its 200 registers make it
// slower (4.23 -> 5.91 ms). MPDG_TANGENT_FIELDS_LPT=1 takes it at every degree, =0 at none.
static bool tangent_fields_lpt(int p)
{
  static const int mode = [] {
    const char *e = getenv("MPDG_TANGENT_FIELDS_LPT");
    return e ? (e[0] == '1' ? 1 : (e[0] == '0' ? 0 : 2)) : 2;
  }();
  return mode == 1 || (mode == 2 && (p == 4 || p == 6));
}

static int ensure_lineark(mpdg_heat *h)
{
  if (!h->tk_dirty) return MPDG_OK;
  TRY(dvec(h, &h->tk, h->n_cells * 4 * h->npt));
  CellArgs<double> a = cell_args<double>(h);
  a.g.q = h->geoq;
  a.Tl = h->T_lin;
  CU(h->tab.coef_lineark(a, h->tk, h->geo, h->stream, h->sm_count));
  ++h->launches;
  h->tk_dirty = false;
  return MPDG_OK;
}

// (re)build the LAW 5 tangent coefficient fields at the current linearisation point
static int ensure_tangent(mpdg_heat *h)
{
  if (!h->tf_dirty) return MPDG_OK;
  TRY(ensure_fields(h));
  TRY(dvec(h, &h->tf, h->n_cells * 8 * h->npt));
  CellArgs<double> a = cell_args<double>(h);
  a.g.q = h->geoq;
  a.cf = h->cf;
  a.Tl = h->T_lin;
  a.To = h->T_old;
  CU(h->tab.coef_tangent(a, h->tf, h->geo, h->stream, h->sm_count));
  ++h->launches;
  h->tf_dirty = false;
  h->tf_f_dirty = true;
  return MPDG_OK;
}

static int ensure_lin(mpdg_heat *h)
{
  if (law_tdep(h) && !h->T_lin)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "temperature-dependent law needs set_linearization");
  if ((h->law == MPDG_LAW_GAS_LIQUID || h->law == MPDG_LAW_GAS_LIQUID_SOLID) && !h->Hf)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "gas-liquid laws need a heaviside field (set_fields)");
  if ((h->law == MPDG_LAW_LIQUID_SOLID || h->law == MPDG_LAW_GAS_LIQUID_SOLID) && h->need_told &&
      !h->T_old)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "liquid-solid law needs temperature_old");
  return MPDG_OK;
}


static bool any_faces(const mpdg_heat *h)
{
  for (int f = 0; f < 6; ++f)
    if (h->btype[f]) return true;
  return false;
}

template <typename T>
static int launch_faces(mpdg_heat *h, int op, T *dst, const T *src, const T *Tl, double *dot,
                        const SolverState *st)
{
  const Tables1D t1 = make_tables(h->n);
  for (int f = 0; f < 6; ++f) {
    if (!h->btype[f]) continue;
    if (op != 1 && !(h->btype[f] & 3)) continue;  // Neumann has no tangent
    FaceArgs<T> a;
    memset(&a, 0, sizeof(a));
    a.d = h->dims;
    a.n = h->n;
    a.face = f;
    a.dir = f / 2;
    a.ea = a.dir == 0 ? 1 : 0;
    a.eb = a.dir == 2 ? 1 : 2;
    a.fixed = (f & 1) ? h->dims.nd[a.dir] - 1 : 0;
    a.type = h->btype[f];
    a.ha = (T)h->hcell[a.ea];
    a.hb = (T)h->hcell[a.eb];
    a.hconv = (T)h->bh[f];
    a.Tinf_c = (T)h->bTc[f];
    a.eps_sigma = (T)(h->beps[f] * kStefanBoltzmann);
    a.Tinf_r4 = (T)std::pow(h->bTr[f], 4);
    a.qn = (T)h->bqn[f];
    for (int q = 0; q < h->n; ++q) {
      a.w[q] = (T)t1.wg[q];
      for (int i = 0; i < h->n; ++i) a.S[q][i] = (T)t1.A[kS][q][i];
    }
    a.src = src;
    a.dst = dst;
    a.Tl = Tl;
    a.dot = dot;
    a.st = st;
    const int blocks = h->dims.m[a.ea] * h->dims.m[a.eb];
    const int threads = ((h->n * h->n + 31) / 32) * 32;
    if (op == 0)
      k_face<T, 0><<<blocks, threads, 0, h->stream>>>(a);
    else if (op == 1)
      k_face<T, 1><<<blocks, threads, 0, h->stream>>>(a);
    else
      k_face<T, 2><<<blocks, threads, 0, h->stream>>>(a);
    ++h->launches;
  }
  CU(cudaGetLastError());
  return MPDG_OK;
}

// dst += J src (FP64); fin/out/st select the fused src.dst reduction
static int op_apply_d(mpdg_heat *h, double *dst, const double *src, int fin, double *out,
                      SolverState *st)
{
  TRY(ensure_dt(h));
  TRY(ensure_lin(h));
  TRY(ensure_fields(h));
  CellArgs<double> a = cell_args<double>(h);
  a.g.q = h->geoq;
  a.cf = h->cf;
  int law = klaw(h);
  if (law == 5 && h->tab.v2_d) {
    TRY(ensure_tangent(h));
    a.cf = h->tf;
    law = 6;
  } else if (law == MPDG_LAW_LINEAR_K && h->tab.coef_lineark && tangent_fields_enabled() &&
             (h->tab.v2_d || (h->geo == 1 && tangent_fields_lpt(h->p)))) {
    // the line-per-thread kernel (p >= 4) takes them on deformed meshes (4 more loads per
    // point against the 6 T_lin sweeps) where that measured faster
    TRY(ensure_lineark(h));
    a.cf = h->tk;
    law = 7;
  }
  a.src = src;
  a.dst = dst;
  a.Tl = h->T_lin;
  a.To = h->T_old;
  a.fin = fin;
  a.out = out;
  a.st = st;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (h->timing) {
    e0 = take_event(h);
    e1 = take_event(h);
    cudaEventRecord(e0, h->stream);
  }
  if (any_faces(h)) {
    TRY(dvec(h, &h->face_dot, 1));
    CU(zero_async(h, h->face_dot, sizeof(double), h->stream));
    TRY(launch_faces<double>(h, 0, dst, src, h->T_lin, fin != FIN_NONE ? h->face_dot : nullptr, st));
    if (fin != FIN_NONE) a.extra_dot = h->face_dot;
  }
  CU(h->tab.vmult_d(a, h->geo, law, h->stream, h->sm_count));
  if (h->timing) {
    cudaEventRecord(e1, h->stream);
    h->ev64.push_back({e0, e1});
  }
  ++h->vm64;
  ++h->launches;
  return MPDG_OK;
}

static int refresh_f32(mpdg_heat *h)
{
  const int64_t N = h->n_dofs;
  if (h->geo == 1 && !h->geoq_f) {
    const int64_t ng = h->n_cells * 7 * h->npt;
    TRY(dvec(h, &h->geoq_f, ng));
    k_cast_f<<<vgrid(h, ng), VT, 0, h->stream>>>(ng, h->geoq, h->geoq_f); ++h->launches;
    CU(cudaGetLastError());
  }
  if (klaw(h) >= 4 && h->cf_f_dirty) {
    TRY(ensure_fields(h));
    const int64_t nc = h->n_cells * 5 * h->npt;
    TRY(dvec(h, &h->cf_f, nc));
    k_cast_f<<<vgrid(h, nc), VT, 0, h->stream>>>(nc, h->cf, h->cf_f); ++h->launches;
    CU(cudaGetLastError());
    h->cf_f_dirty = false;
  }
  // T_lin in FP32 for the temperature-dependent laws and the radiation faces' tangent
  bool radiation = false;
  for (int f = 0; f < 6; ++f) radiation = radiation || (h->btype[f] & MPDG_BC_RADIATION);
  if (h->lin_f_dirty && h->T_lin && (law_tdep(h) || radiation)) {
    TRY(dvec(h, &h->T_lin_f, N));
    TRY(dvec(h, &h->T_old_f, N));
    k_cast_f<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->T_lin, h->T_lin_f); ++h->launches;
    if (h->T_old) {
      k_cast_f<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->T_old, h->T_old_f);
      ++h->launches;
    }
    CU(cudaGetLastError());
  }
  h->lin_f_dirty = false;
  return MPDG_OK;
}

// The FP32 Picard operator on the tensor cores (TF32 operands, FP32 accumulation) where the
// kernel exists (uniform box, FE_Q(3)), when MPDG_PICARD_TC=1 or mpdg_heat_set_picard_tensor_cores
// asks for it; the default is the CUDA-core kernel, which measured faster (the operator is bound
// by its gather/scatter path, not by the contractions the tensor cores take over)
static bool picard_tc_on(const mpdg_heat *h)
{
  static const int env_on = [] {
    const char *e = getenv("MPDG_PICARD_TC");
    return (e && e[0] == '1') ? 1 : 0;
  }();
  const int on = h->picard_tc >= 0 ? h->picard_tc : env_on;
  return on && h->geo == 0 && h->p == 3 && h->tab.vmult_picard_tc != nullptr;
}

// The Picard operator with k(T_lin(q)) interpolated in the kernel from the gathered FP32 T_lin
// instead of read from the stored per-point field (LAW 8; the same operator for the linear-k
// law, which is affine in T): MPDG_PICARD_NODAL=1, register-resident kernel degrees only
static bool picard_nodal(const mpdg_heat *h)
{
  static const int env_on = [] {
    const char *e = getenv("MPDG_PICARD_NODAL");
    return (e && e[0] == '1') ? 1 : 0;
  }();
  return env_on && h->law == MPDG_LAW_LINEAR_K && h->tab.v2_f;
}

static int ensure_picard_tc(mpdg_heat *h)
{
  if (!h->gmat_tc) {
    std::vector<float> g(2 * optc::kGFloats);
    optc::build_gmat(g.data());
    TRY(dalloc(h, (void **)&h->gmat_tc, 2 * optc::kGBytes));
    CU(cudaMemcpy(h->gmat_tc, g.data(), 2 * optc::kGBytes, cudaMemcpyHostToDevice));
  }
  if (!h->tc_err_host) {
    if (cudaHostAlloc((void **)&h->tc_err_host, sizeof(int), cudaHostAllocMapped) != cudaSuccess)
      return fail(MPDG_ERR_OUT_OF_MEMORY, "cudaHostAlloc");
    *h->tc_err_host = 0;
    CU(cudaHostGetDevicePointer((void **)&h->tc_err_map, h->tc_err_host, 0));
  }
  if (*(volatile int *)h->tc_err_host)
    return fail(MPDG_ERR_CUDA, "tensor-core Picard operator: an MMA wait timed out");
  return MPDG_OK;
}

// src_rows (optional): the operand in the cell-row layout (FP32 Picard operator of FE_Q(3),
// no boundary-face terms); src is then not read
static int op_apply_f(mpdg_heat *h, float *dst, const float *src, SolverState *st,
                      bool picard = false, const float *src_rows = nullptr)
{
  TRY(ensure_dt(h));
  TRY(ensure_lin(h));
  TRY(ensure_fields(h));
  TRY(refresh_f32(h));
  CellArgs<float> a = cell_args<float>(h);
  a.kq = h->kq;
  a.cf = h->cf_f;
  int law = picard ? (picard_nodal(h) ? 8 : 3) : klaw(h);
  if (law == 5 && h->tab.v2_f) {
    TRY(ensure_tangent(h));
    const int64_t nt = h->n_cells * 8 * h->npt;
    if (h->tf_f_dirty) {
      TRY(dvec(h, &h->tf_f, nt));
      k_cast_f<<<vgrid(h, nt), VT, 0, h->stream>>>(nt, h->tf, h->tf_f); ++h->launches;
      CU(cudaGetLastError());
      h->tf_f_dirty = false;
    }
    a.cf = h->tf_f;
    law = 6;
  }
  a.g.q = h->geoq_f;
  a.src = src;
  a.dst = dst;
  a.Tl = h->T_lin_f;
  a.To = h->T_old_f;
  a.st = st;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (h->timing) {
    e0 = take_event(h);
    e1 = take_event(h);
    cudaEventRecord(e0, h->stream);
  }
  const bool tc = law == 3 && picard_tc_on(h);
  if (src_rows && (law != 3 || tc || any_faces(h) || !h->tab.vmult_picard_rows))
    return fail(MPDG_ERR_INVALID_ARGUMENT,
                "cell-row operand: FP32 Picard operator of FE_Q(3) without boundary faces only");
  if (tc) TRY(ensure_picard_tc(h));
  if (any_faces(h)) TRY(launch_faces<float>(h, 0, dst, src, h->T_lin_f, nullptr, st));
  if (src_rows) {
    a.src = src_rows;
    a.fin = FIN_NONE;
    CU(h->tab.vmult_picard_rows(a, h->geo, h->stream, h->sm_count));
  } else if (tc) {
    CU(h->tab.vmult_picard_tc(a, h->gmat_tc, h->tc_err_map, h->stream, h->sm_count));
  } else {
    CU(h->tab.vmult_f(a, h->geo, law, h->stream, h->sm_count));
  }
  if (h->timing) {
    cudaEventRecord(e1, h->stream);
    h->ev32.push_back({e0, e1});
  }
  ++h->vm32;
  ++h->launches;
  return MPDG_OK;
}

// copies n 4-byte words into mapped page-locked host memory: the stores travel over the host
// link from the SMs, so a read of a few words does not queue behind a bulk copy (the host
// step's T_old download during the solve) on the device-to-host copy engine
__global__ void k_read_words(const unsigned *__restrict__ src, unsigned *dst, int n)
{
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

static int read_to_host(mpdg_heat *h, void *mapped, const void *dev, size_t bytes)
{
  k_read_words<<<1, 256, 0, h->stream>>>((const unsigned *)dev, (unsigned *)mapped,
                                         (int)(bytes / sizeof(unsigned)));
  ++h->launches;
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(h->stream));
  return MPDG_OK;
}
static_assert(sizeof(SolverState) % sizeof(unsigned) == 0, "SolverState is read in words");

static int poll(mpdg_heat *h) { return read_to_host(h, h->st_map, h->st, sizeof(SolverState)); }

static int norms(mpdg_heat *h, const double *a, const double *b, double *aa, double *ab)
{
  const int64_t N = h->n_dofs;
  k_norms<<<vgrid(h, N), VT, 0, h->stream>>>(N, a, b, h->partials, h->counter, h->scal); ++h->launches;
  CU(cudaGetLastError());
  TRY(read_to_host(h, h->scal_map, h->scal, 2 * sizeof(double)));
  if (aa) *aa = h->scal_host[0];
  if (ab) *ab = h->scal_host[1];
  return MPDG_OK;
}

static int ensure_workspace(mpdg_heat *h)
{
  const int64_t N = h->n_dofs;
  TRY(dvec(h, &h->r, N));
  TRY(dvec(h, &h->pv, N));
  TRY(dvec(h, &h->Ap, N));
  return MPDG_OK;
}

static int ensure_workspace_f32(mpdg_heat *h)
{
  const int64_t N = h->n_dofs;
  TRY(dvec(h, &h->z, N));
  TRY(dvec(h, &h->r32, N));
  TRY(dvec(h, &h->x32, N));
  TRY(dvec(h, &h->d32, N));
  TRY(dvec(h, &h->Ax32, N));
  TRY(dvec(h, &h->inv_diag_f, N));
  return MPDG_OK;
}

__global__ void k_scale_copy(int64_t N, double *dst, const double *__restrict__ src, double a)
{
  GRID_STRIDE(i, N) dst[i] = a * src[i];
}

// Ap = A x at the start of a solve: zero when the solve starts from x = 0 (x_zero), the
// step's precomputed A x when it gave one (x_Ax, used once), else one operator application
static int initial_Ax(mpdg_heat *h, const double *x)
{
  const int64_t N = h->n_dofs;
  if (h->x_Ax) {
    k_scale_copy<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->Ap, h->x_Ax, h->x_Ax_scale);
    ++h->launches;
    CU(cudaGetLastError());
  } else {
    CU(zero_async(h, h->Ap, sizeof(double) * N, h->stream));
    if (!h->x_zero) TRY(op_apply_d(h, h->Ap, x, FIN_NONE, nullptr, nullptr));
  }
  h->x_Ax = nullptr;
  h->x_zero = false;
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// CG (FP64, identity or Jacobi); record = Lanczos history for eigenvalues
// ---------------------------------------------------------------------------
static int cg_jacobi(mpdg_heat *h, const mpdg_solver_params *prm, double *x, const double *b,
                     const double *D, int record, mpdg_solve_stats *stats)
{
  const int64_t N = h->n_dofs;
  TRY(ensure_workspace(h));
  const int g = vgrid(h, N);
  TRY(initial_Ax(h, x));
  k_cg_init<<<g, VT, 0, h->stream>>>(N, b, h->r, h->pv, h->Ap, D, h->st, h->partials, h->counter,
                                      prm->rel_tolerance, prm->abs_tolerance,
                                      prm->tol_reference_norm, prm->max_iterations, record); ++h->launches;
  CU(cudaGetLastError());
  TRY(poll(h));
  const double res0 = h->st_host->res0;
  int chunk = 4;
  while (!h->st_host->done) {
    for (int c = 0; c < chunk; ++c) {
      TRY(op_apply_d(h, h->Ap, h->pv, FIN_CG_ALPHA, nullptr, h->st));
      k_cg_update_xr<<<g, VT, 0, h->stream>>>(N, x, h->r, h->pv, h->Ap, D, h->st, h->partials,
                                              h->counter); ++h->launches;
      k_cg_update_p<<<g, VT, 0, h->stream>>>(N, h->r, h->pv, h->Ap, D, h->st); ++h->launches;
    }
    CU(cudaGetLastError());
    TRY(poll(h));
    chunk = std::min(chunk * 2, 64);
  }
  if (stats) {
    stats->iterations = h->st_host->it;
    stats->status = h->st_host->done == 1 ? MPDG_OK : h->st_host->status;
    stats->initial_residual = res0;
    stats->final_residual = h->st_host->res;
    stats->true_residual = h->st_host->res;
  }
  return MPDG_OK;
}

// Lanczos estimate of the extreme eigenvalues of D^-1 J
static double tridiag_eig(int m, const double *d, const double *e, int which)
{
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < m; ++i) {
    const double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i < m - 1 ? std::fabs(e[i]) : 0.0);
    lo = std::min(lo, d[i] - r);
    hi = std::max(hi, d[i] + r);
  }
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    int cnt = 0;
    double q = d[0] - mid;
    if (q < 0) ++cnt;
    for (int i = 1; i < m; ++i) {
      if (q == 0.0) q = 1e-300;
      q = d[i] - mid - e[i - 1] * e[i - 1] / q;
      if (q < 0) ++cnt;
    }
    if (cnt > which)
      hi = mid;
    else
      lo = mid;
  }
  return 0.5 * (lo + hi);
}

static int estimate_eigenvalues(mpdg_heat *h, int n_it, double *lmin, double *lmax)
{
  const int64_t N = h->n_dofs;
  n_it = std::max(2, std::min(n_it, 64));
  TRY(dvec(h, &h->w3, N));
  TRY(dvec(h, &h->z, N));
  k_masked_random<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->dims, h->w3); ++h->launches;
  CU(zero_async(h, h->z, sizeof(double) * N, h->stream));
  mpdg_solver_params prm;
  mpdg_solver_params_default(&prm);
  prm.max_iterations = n_it;
  prm.rel_tolerance = 0.0;
  prm.abs_tolerance = 0.0;
  // the Lanczos CG starts from z = 0; the caller's own zero-start hint is kept for its solve
  const bool keep_x_zero = h->x_zero;
  h->x_zero = true;
  const int rc_cg = cg_jacobi(h, &prm, h->z, h->w3, h->inv_diag, 1, nullptr);
  h->x_zero = keep_x_zero;
  TRY(rc_cg);
  const SolverState &s = *h->st_host;
  const int m = std::min(s.it, 64);
  if (m < 1) {
    *lmin = *lmax = 1.0;
    return MPDG_OK;
  }
  std::vector<double> d(m), e(m, 0.0);
  for (int j = 0; j < m; ++j) {
    d[j] = 1.0 / s.hist_alpha[j] + (j > 0 ? s.hist_beta[j - 1] / s.hist_alpha[j - 1] : 0.0);
    if (j + 1 < m) e[j] = std::sqrt(s.hist_beta[j]) / s.hist_alpha[j];
  }
  *lmin = tridiag_eig(m, d.data(), e.data(), 0);
  *lmax = tridiag_eig(m, d.data(), e.data(), m - 1);
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// FP32 p-multigrid preconditioner. Levels: the solver's FE_Q(p) operator, FE_Q(1)
// on the same mesh (p > 1), then FE_Q(1) on meshes coarsened by two per direction
// while every cell count stays even and its half >= mg_min_cells. Each coarse
// level is a child handle with the same material, boundary terms and Dirichlet
// faces, linearised at the injection of the fine linearisation point; its operator
// is the same FP32 form as the fine one (Picard when the outer solve uses it).
// Transfers are separable tensor products of the 1D interpolation between nested
// node sets (the GLL nodes of FE_Q(p) for the p step, midpoints for the h step),
// the restriction its transpose. Smoother: Chebyshev-Jacobi over
// [upper / mg_smoothing_range, upper] with upper = cheb_max_factor * lambda_max of
// D^-1 A from a Lanczos estimate per level; the coarsest level runs
// mg_coarse_degree steps over [lambda_min, upper].
// ---------------------------------------------------------------------------
static void release(mpdg_heat *h);
static std::vector<double> box_vertices(const mpdg_mesh_desc &desc);
static int create_impl(const mpdg_mesh_desc *desc, int device, const std::vector<double> *verts,
                       mpdg_heat **out);
static int compute_diag(mpdg_heat *h, double *d, bool invert = true);

static void cheb_coefficients(double theta, double delta, int k, std::vector<float> &c1,
                              std::vector<float> &c2)
{
  const double sigma = theta / delta;
  c1.assign(k + 1, 0.f);
  c2.assign(k + 1, 0.f);
  double rho0 = 1.0 / sigma;
  for (int j = 1; j <= k; ++j) {
    const double rho1 = 1.0 / (2.0 * sigma - rho0);
    c1[j] = (float)(rho1 * rho0);
    c2[j] = (float)(2.0 * rho1 / delta);
    rho0 = rho1;
  }
}

static Dims3 nodal_dims(const mpdg_heat *h) { return Dims3{{h->dims.nd[0], h->dims.nd[1], h->dims.nd[2]}}; }

// inverse diagonal of the FP32 Picard operator into h->inv_diag_f (h->kq current);
// h->d32 serves as the accumulator (its content is dead outside a preconditioner call)
static int picard_inverse_diagonal(mpdg_heat *h)
{
  const int64_t N = h->n_dofs;
  TRY(ensure_dt(h));
  TRY(ensure_workspace_f32(h));
  TRY(refresh_f32(h));
  CU(zero_async(h, h->d32, sizeof(float) * N, h->stream));
  CellArgs<float> a = cell_args<float>(h);
  a.kq = h->kq;
  a.g.q = h->geoq_f;
  a.dst = h->d32;
  CU(h->tab.diag_picard(a, h->geo, h->stream, h->sm_count));
  ++h->launches;
  if (any_faces(h)) TRY(launch_faces<float>(h, 2, h->d32, nullptr, h->T_lin_f, nullptr, nullptr));
  k_invert_diag_f<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->d32, h->inv_diag_f);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

static int mg_build(mpdg_heat *h, const mpdg_solver_params *prm)
{
  if (!h->mg.empty() && h->mg_min_cells == prm->mg_min_cells) return MPDG_OK;
  for (MGLevel &lv : h->mg)
    if (lv.own && lv.h) {
      release(lv.h);
      delete lv.h;
    }
  h->mg.clear();
  h->mg_min_cells = prm->mg_min_cells;
  MGLevel l0;
  l0.h = h;
  l0.b = h->r32;
  l0.x = h->x32;
  l0.d = h->d32;
  l0.Ax = h->Ax32;
  h->mg.push_back(l0);
  mpdg_mesh_desc cur = h->desc;
  std::vector<double> cur_verts;
  if (h->geo == 1) cur_verts = box_vertices(h->desc);
  auto add_child = [&](int ratio, const float *xi, const mpdg_mesh_desc &d,
                       const std::vector<double> *verts) -> int {
    mpdg_heat *c = nullptr;
    TRY(create_impl(&d, h->device, verts, &c));
    h->mg.back().ratio = ratio;
    for (int a = 0; a < ratio && a < 8; ++a) h->mg.back().xi[a] = xi[a];
    MGLevel lv;
    lv.h = c;
    lv.own = true;
    h->mg.push_back(lv);
    MGLevel &L = h->mg.back();
    c->stream = h->stream;
    c->latent = h->latent;
    c->acap = h->acap;
    TRY(mpdg_heat_set_material(c, &h->mat));
    for (int f = 0; f < 6; ++f) {
      c->btype[f] = h->btype[f];
      c->bh[f] = h->bh[f];
      c->bTc[f] = h->bTc[f];
      c->beps[f] = h->beps[f];
      c->bTr[f] = h->bTr[f];
      c->bqn[f] = h->bqn[f];
    }
    TRY(ensure_workspace_f32(c));
    TRY(dvec(c, &c->inv_diag, c->n_dofs));
    TRY(dvec(c, &L.Tl, c->n_dofs));
    TRY(dvec(c, &L.To, c->n_dofs));
    L.b = c->r32;
    L.x = c->x32;
    L.d = c->d32;
    L.Ax = c->Ax32;
    CU(zero_async(h, L.Ax, sizeof(float) * c->n_dofs, h->stream));
    return MPDG_OK;
  };
  if (h->p > 1) {
    const Tables1D t = make_tables(h->n);
    float xi[8];
    for (int a = 0; a < h->p && a < 8; ++a) xi[a] = (float)t.xl[a];
    mpdg_mesh_desc d = cur;
    d.degree = 1;
    TRY(add_child(h->p, xi, d, h->geo == 1 ? &cur_verts : nullptr));
    cur = d;
  }
  for (;;) {
    bool ok = true;
    for (int e = 0; e < 3; ++e)
      if (cur.cells[e] % 2 != 0 || cur.cells[e] / 2 < std::max(1, prm->mg_min_cells)) ok = false;
    if (!ok) break;
    mpdg_mesh_desc d = cur;
    d.degree = 1;
    for (int e = 0; e < 3; ++e) d.cells[e] = cur.cells[e] / 2;
    std::vector<double> cv;
    if (h->geo == 1) {
      // vertices of the coarse mesh = every second vertex of the current one
      cv.resize((size_t)3 * (d.cells[0] + 1) * (d.cells[1] + 1) * (d.cells[2] + 1));
      for (int c = 0; c <= d.cells[2]; ++c)
        for (int b = 0; b <= d.cells[1]; ++b)
          for (int a = 0; a <= d.cells[0]; ++a) {
            const int64_t vc = a + (int64_t)(d.cells[0] + 1) * (b + (int64_t)(d.cells[1] + 1) * c);
            const int64_t vf = 2 * a + (int64_t)(cur.cells[0] + 1) *
                                         (2 * b + (int64_t)(cur.cells[1] + 1) * 2 * c);
            for (int e = 0; e < 3; ++e) cv[3 * vc + e] = cur_verts[3 * vf + e];
          }
    }
    const float xi[2] = {0.f, 0.5f};
    TRY(add_child(2, xi, d, h->geo == 1 ? &cv : nullptr));
    cur = d;
    cur_verts.swap(cv);
  }
  if (h->mg.size() < 2)
    return fail(MPDG_ERR_INVALID_ARGUMENT,
                "multigrid needs degree > 1 or even cell counts with halves >= mg_min_cells");
  // transfer scratch: the largest x-pass and y-pass intermediates
  int64_t n1 = 0, n2 = 0;
  for (size_t l = 0; l + 1 < h->mg.size(); ++l) {
    const Dims3 F = nodal_dims(h->mg[l].h), C = nodal_dims(h->mg[l + 1].h);
    n1 = std::max(n1, (int64_t)C.n[0] * F.n[1] * F.n[2]);
    n2 = std::max(n2, (int64_t)C.n[0] * C.n[1] * F.n[2]);
  }
  TRY(dvec(h, &h->mg_t1, n1));
  TRY(dvec(h, &h->mg_t2, n2));
  return MPDG_OK;
}

static int estimate_eigenvalues(mpdg_heat *h, int n_it, double *lmin, double *lmax);

// per solve: linearise the coarse levels at the injected point, their conductivity
// fields, inverse diagonals and (first time, or without reuse) smoothing intervals
static int mg_setup(mpdg_heat *h, const mpdg_solver_params *prm, bool picard)
{
  const int L = (int)h->mg.size();
  const int s = std::max(1, prm->mg_smoothing_degree);
  for (int l = 0; l < L; ++l) {
    MGLevel &v = h->mg[l];
    mpdg_heat *c = v.h;
    if (l > 0) {
      const MGLevel &f = h->mg[l - 1];
      const double *fT = l == 1 ? h->T_lin : f.Tl;
      const double *fTo = l == 1 ? h->T_old : (f.h->T_old ? f.To : nullptr);
      const Dims3 F = nodal_dims(f.h), Cd = nodal_dims(c);
      if (fT) {
        k_inject<<<vgrid(c, Cd.size()), VT, 0, h->stream>>>(F, Cd, f.ratio, fT, v.Tl); ++h->launches;
      }
      if (fTo) {
        k_inject<<<vgrid(c, Cd.size()), VT, 0, h->stream>>>(F, Cd, f.ratio, fTo, v.To); ++h->launches;
      }
      CU(cudaGetLastError());
      if (c->dt != h->dt) {
        c->dt = h->dt;
        c->eig_valid = false;
      }
      c->T_lin = fT ? v.Tl : nullptr;
      c->T_old = fTo ? v.To : nullptr;
      c->lin_f_dirty = true;
      c->tf_dirty = true;
      c->tk_dirty = true;
      TRY(refresh_f32(c));
      if (picard) {
        TRY(dvec(c, &c->kq, c->n_cells * c->npt));
        CellArgs<double> a = cell_args<double>(c);
        a.Tl = c->T_lin;
        CU(c->tab.conductivity_q(a, c->kq, c->law, h->stream, c->sm_count));
        ++h->launches;
      }
      const bool estimate = !c->eig_valid || !prm->cheb_eig_reuse;
      if (estimate || !picard) {
        // FP64 tangent diagonal: for the Lanczos estimate, and as the smoother's
        // diagonal when the levels apply the tangent itself
        TRY(compute_diag(c, c->inv_diag));
        c->diag_valid = true;
      }
      if (estimate) {
        TRY(estimate_eigenvalues(c, prm->cheb_eig_iterations, &c->eig_min, &c->eig_max));
        c->eig_valid = true;
      }
    }
    // the smoother's Jacobi diagonal: of the operator the level applies
    if (picard) {
      TRY(picard_inverse_diagonal(c));
      if (l == 0) h->diag_f_dirty = true;  // inv_diag_f no longer mirrors the FP64 diagonal
    } else if (l > 0) {
      k_cast_f<<<vgrid(c, c->n_dofs), VT, 0, h->stream>>>(c->n_dofs, c->inv_diag, c->inv_diag_f);
      ++h->launches;
      CU(cudaGetLastError());
    }
    const double upper = prm->cheb_max_factor * c->eig_max;
    double lower = upper / std::max(1.5, prm->mg_smoothing_range);
    v.pre = v.post = s;
    if (l == 0) {
      if (prm->mg_fine_pre_steps >= 0) v.pre = prm->mg_fine_pre_steps;
      if (prm->mg_fine_post_steps >= 0) v.post = prm->mg_fine_post_steps;
    }
    if (l == L - 1) {
      lower = std::min(lower, std::max(c->eig_min, 1e-6 * upper));
      v.pre = std::max(1, prm->mg_coarse_degree);
      v.post = 0;
    }
    v.theta = 0.5 * (upper + lower);
    v.delta = 0.5 * (upper - lower);
    cheb_coefficients(v.theta, v.delta, std::max(v.pre, v.post), v.c1, v.c2);
  }
  return MPDG_OK;
}

// coarse = R (fine_b - fine_Ax)
static int mg_restrict(mpdg_heat *h, int l, const float *fine_Ax, const float *fine_b,
                       float *coarse)
{
  const MGLevel &f = h->mg[l], &c = h->mg[l + 1];
  const Dims3 F = nodal_dims(f.h), C = nodal_dims(c.h);
  const Dims3 D1{{C.n[0], F.n[1], F.n[2]}}, D2{{C.n[0], C.n[1], F.n[2]}};
  Transfer1D t;
  t.r = f.ratio;
  for (int a = 0; a < 8; ++a) t.xi[a] = f.xi[a];
  k_restrict_axis<<<vgrid(h, D1.size()), VT, 0, h->stream>>>(0, F, D1, t, fine_Ax, fine_b,
                                                             h->mg_t1, c.h->dims, 0, h->st);
  k_restrict_axis<<<vgrid(h, D2.size()), VT, 0, h->stream>>>(1, D1, D2, t, h->mg_t1, nullptr,
                                                             h->mg_t2, c.h->dims, 0, h->st);
  k_restrict_axis<<<vgrid(h, C.size()), VT, 0, h->stream>>>(2, D2, C, t, h->mg_t2, nullptr, coarse,
                                                            c.h->dims, 1, h->st);
  h->launches += 3;
  CU(cudaGetLastError());
  return MPDG_OK;
}

// fine += P coarse (constrained rows untouched); zero_fine (fine-shaped) is set to zero;
// fine in fine_rows' cell rows instead when fine_rows.rows is set
static int mg_prolong_add(mpdg_heat *h, int l, const float *coarse, float *fine, float *zero_fine,
                          CellRows fine_rows = CellRows())
{
  const MGLevel &f = h->mg[l], &c = h->mg[l + 1];
  const Dims3 F = nodal_dims(f.h), C = nodal_dims(c.h);
  const Dims3 E2{{C.n[0], C.n[1], F.n[2]}}, E1{{C.n[0], F.n[1], F.n[2]}};
  Transfer1D t;
  t.r = f.ratio;
  for (int a = 0; a < 8; ++a) t.xi[a] = f.xi[a];
  k_prolong_axis<false><<<vgrid(h, E2.size()), VT, 0, h->stream>>>(2, C, E2, t, coarse, h->mg_t2, 0,
                                                            f.h->dims, 0, nullptr, h->st,
                                                            CellRows());
  k_prolong_axis<false><<<vgrid(h, E1.size()), VT, 0, h->stream>>>(1, E2, E1, t, h->mg_t2, h->mg_t1, 0,
                                                            f.h->dims, 0, nullptr, h->st,
                                                            CellRows());
  auto kp = fine_rows.rows ? k_prolong_axis<true> : k_prolong_axis<false>;
  kp<<<vgrid(h, F.size()), VT, 0, h->stream>>>(0, E1, F, t, h->mg_t1, fine, 1,
                                                           f.h->dims, 1, zero_fine, h->st,
                                                           fine_rows);
  h->launches += 3;
  CU(cudaGetLastError());
  return MPDG_OK;
}

template <bool ROWS>
__global__ void k_cheb_step(int64_t N, const float *__restrict__ r32, float *x32, float *d32,
                            float *Ax32, const float *__restrict__ D32, float c1, float c2,
                            const SolverState *st, CellRows xr);
template <bool ROWS>
__global__ void k_cheb_last(int64_t N, const float *__restrict__ r32, const float *__restrict__ x32,
                            const float *__restrict__ d32, float *Ax32,
                            const float *__restrict__ D32, float c1, float c2,
                            const double *__restrict__ r, const double *__restrict__ Ap, double *z,
                            SolverState *st, double *partials, unsigned *counter, CellRows xr);

// one V-cycle on the FP32 residual in level 0's b (= r32), whose first smoothing step
// (x = d = D b / theta_0) the caller has taken; ends with z = x (FP64) and the dots of
// the flexible CG, like the last Chebyshev step. Level 0's iterate is in the handle's cell
// rows while rows_on (the caller's first step wrote it there).
static int mg_vcycle(mpdg_heat *h, bool picard)
{
  const int L = (int)h->mg.size();
  SolverState *st = h->st;
  for (int l = 0; l < L; ++l) {
    MGLevel &v = h->mg[l];
    mpdg_heat *c = v.h;
    const int64_t N = c->n_dofs;
    const int g = vgrid(c, N);
    const CellRows xr = l == 0 ? cell_rows_of(h) : CellRows();
    if (l > 0) {
      k_cheb_init<<<g, VT, 0, h->stream>>>(N, v.b, v.x, v.d, c->inv_diag_f, (float)(1.0 / v.theta),
                                           st);
      ++h->launches;
    }
    for (int j = 1; j <= v.pre; ++j) {
      TRY(op_apply_f(c, v.Ax, v.x, st, picard, xr.rows));
      (xr.rows ? k_cheb_step<true> : k_cheb_step<false>)<<<g, VT, 0, h->stream>>>(
        N, v.b, v.x, v.d, v.Ax, c->inv_diag_f, v.c1[j],
                                           v.c2[j], st, xr);
      ++h->launches;
    }
    if (l == L - 1) break;
    // residual b - A x restricted (formed inside the first pass); Ax is reset to zero by
    // the last prolongation pass on the way back up
    TRY(op_apply_f(c, v.Ax, v.x, st, picard, xr.rows));
    TRY(mg_restrict(h, l, v.Ax, v.b, h->mg[l + 1].b));
  }
  for (int l = L - 2; l >= 0; --l) {
    MGLevel &v = h->mg[l];
    mpdg_heat *c = v.h;
    const int64_t N = c->n_dofs;
    const int g = vgrid(c, N);
    const CellRows xr = l == 0 ? cell_rows_of(h) : CellRows();
    TRY(mg_prolong_add(h, l, h->mg[l + 1].x, v.x, v.Ax, xr));
    // post-smoothing: the Chebyshev recurrence restarted from the corrected iterate
    for (int j = 0; j <= v.post; ++j) {
      TRY(op_apply_f(c, v.Ax, v.x, st, picard, xr.rows));
      const float c1 = j == 0 ? 0.f : v.c1[j];
      const float c2 = j == 0 ? (float)(1.0 / v.theta) : v.c2[j];
      if (l == 0 && j == v.post) {
        (xr.rows ? k_cheb_last<true> : k_cheb_last<false>)<<<g, VT, 0, h->stream>>>(
          N, v.b, v.x, v.d, v.Ax, c->inv_diag_f, c1, c2, h->r,
                                             h->Ap, h->z, st, h->partials, h->counter, xr);
      } else {
        (xr.rows ? k_cheb_step<true> : k_cheb_step<false>)<<<g, VT, 0, h->stream>>>(
          N, v.b, v.x, v.d, v.Ax, c->inv_diag_f, c1, c2, st,
                                             xr);
      }
      ++h->launches;
    }
  }
  CU(cudaGetLastError());
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// CUDA graph of one solver iteration
//
// An iteration of the mixed-precision CG issues ~250 launches (the FP64 operator, the vector
// updates and the V-cycle's smoothing, transfer and coarse-level kernels, many of them a few
// microseconds long), the same sequence with the same arguments in every iteration of a
// solve. It is recorded once per solve into a graph and replayed. Recording runs on a
// private stream (the handle's stream may be the legacy default stream, which cannot be
// captured) with every level's kernels redirected to it; the replay goes to the handle's
// stream. The executable graph is kept and updated in place by the next solve's recording
// when the topology is unchanged. Kernels test the device-side `done` flag, so a replay
// after convergence exits at once, as the direct launches do. MPDG_GRAPHS=0 launches directly.
// ---------------------------------------------------------------------------
static bool graphs_enabled()
{
  static const int on = [] {
    const char *e = getenv("MPDG_GRAPHS");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return on != 0;
}

static void set_level_streams(mpdg_heat *h, cudaStream_t s)
{
  h->stream = s;
  for (MGLevel &lv : h->mg)
    if (lv.h) lv.h->stream = s;
}

// record `body` into h->body_exec; false (nothing recorded, nothing launched) on any failure
template <typename F>
static bool record_body(mpdg_heat *h, F &&body)
{
  if (!h->cap_stream &&
      cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
    h->cap_stream = nullptr;
    cudaGetLastError();
    return false;
  }
  const cudaStream_t orig = h->stream;
  // counters of every level before recording (the coarse levels count their own launches)
  std::vector<std::array<int64_t, 3>> before;
  for (MGLevel &lv : h->mg)
    if (lv.h && lv.h != h) before.push_back({lv.h->launches, lv.h->vm64, lv.h->vm32});
  const int64_t l0 = h->launches, a0 = h->vm64, b0 = h->vm32;
  set_level_streams(h, h->cap_stream);
  cudaGraph_t graph = nullptr;
  bool ok = cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    const int rc = body();
    ok = cudaStreamEndCapture(h->cap_stream, &graph) == cudaSuccess && rc == MPDG_OK && graph;
  }
  set_level_streams(h, orig);
  // a replay is accounted on this handle: what all levels recorded, which did not run
  h->body_launches = h->launches - l0;
  h->body_vm64 = h->vm64 - a0;
  h->body_vm32 = h->vm32 - b0;
  h->launches = l0;
  h->vm64 = a0;
  h->vm32 = b0;
  size_t i = 0;
  for (MGLevel &lv : h->mg)
    if (lv.h && lv.h != h) {
      h->body_launches += lv.h->launches - before[i][0];
      h->body_vm64 += lv.h->vm64 - before[i][1];
      h->body_vm32 += lv.h->vm32 - before[i][2];
      lv.h->launches = before[i][0];
      lv.h->vm64 = before[i][1];
      lv.h->vm32 = before[i][2];
      ++i;
    }
  if (ok && h->body_exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(h->body_exec, graph, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(h->body_exec);
      h->body_exec = nullptr;
    }
  }
  if (ok && !h->body_exec &&
      cudaGraphInstantiate(&h->body_exec, graph, 0) != cudaSuccess) {
    h->body_exec = nullptr;
    ok = false;
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();  // a failed recording leaves a non-sticky error behind
  return ok;
}

// The fine level's Chebyshev iterate in the cell-row layout (opt-in, MPDG_PICARD_ROWS=1), so
// that the FP32 Picard operator gathers each cell row with one vector load: FE_Q(3), the Picard
// operator on the CUDA cores (not the nodal-conductivity or tensor-core forms, not the
// packed-pair kernel), no boundary faces (their kernel reads the lexicographic operand), fewer
// than 2^32 DoFs. Both layouts compute the same iterates. The operator is faster from cell rows
// (0.60 against 0.69 ms at 57 M DoFs), but the Chebyshev, update and prolongation kernels that
// keep the iterate there cost more than that (a benchmark step 86.1 against 84.3 ms).
static bool picard_rows_env()
{
  static const int on = [] {
    const char *e = getenv("MPDG_PICARD_ROWS");
    const char *pk = getenv("MPDG_FP32_PACKED");
    return (e && e[0] == '1' && !(pk && pk[0] == '1')) ? 1 : 0;
  }();
  return on != 0;
}
static int enable_cell_rows(mpdg_heat *h, bool picard)
{
  h->rows_on = false;
  if (!picard || !picard_rows_env() || !h->tab.vmult_picard_rows || picard_nodal(h) ||
      picard_tc_on(h) || any_faces(h) || h->n_dofs >= ((int64_t)1 << 32))
    return MPDG_OK;
  TRY(dvec(h, &h->x32_rows, cell_rows_size(h)));
  h->rows_on = true;
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// FP64 flexible CG with the FP32 Chebyshev-Jacobi or p-multigrid preconditioner
// ---------------------------------------------------------------------------
static int distribute(mpdg_heat *h, double *u);

// the preconditioner's set-up at the current linearisation point: FP32 copies, the Picard
// conductivity field, the eigenvalue estimate (first time, or without reuse) and the multigrid
// levels. It needs no right-hand side, so a time step issues it before it waits for the
// source's upload (h->mixed_ready: the next cg_chebyshev call skips it)
static int mixed_prepare(mpdg_heat *h, const mpdg_solver_params *prm)
{
  const int64_t N = h->n_dofs;
  const bool use_mg = prm->preconditioner == MPDG_PRECOND_MG_F32;
  if (use_mg && klaw(h) >= 4)
    return fail(MPDG_ERR_INVALID_ARGUMENT,
                "multigrid preconditioner: not available with the gas-liquid laws or a velocity field");
  const bool picard = prm->cheb_picard && h->law == MPDG_LAW_LINEAR_K && h->tab.conductivity_q;
  const bool need_diag = !(use_mg && picard) || !h->eig_valid || !prm->cheb_eig_reuse;
  if (need_diag && !h->diag_valid)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "preconditioner not updated");
  if (prm->cheb_degree < 1) return fail(MPDG_ERR_INVALID_ARGUMENT, "cheb_degree < 1");
  if (prm->preconditioner == MPDG_PRECOND_MG_F32 &&
      (prm->mg_smoothing_degree < 1 || prm->mg_coarse_degree < 1 || !(prm->mg_smoothing_range > 1.0)))
    return fail(MPDG_ERR_INVALID_ARGUMENT, "multigrid: smoothing degrees >= 1, range > 1");
  TRY(ensure_workspace(h));
  TRY(ensure_workspace_f32(h));
  TRY(refresh_f32(h));
  if (h->diag_f_dirty && !(use_mg && picard)) {
    k_cast_f<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->inv_diag, h->inv_diag_f); ++h->launches;
    CU(cudaGetLastError());
    h->diag_f_dirty = false;
  }
  if (picard) {
    TRY(dvec(h, &h->kq, h->n_cells * h->npt));
    CellArgs<double> a = cell_args<double>(h);
    a.Tl = h->T_lin;
    CU(h->tab.conductivity_q(a, h->kq, h->law, h->stream, h->sm_count));
    ++h->launches;
  }
  if (!h->eig_valid || !prm->cheb_eig_reuse) {
    TRY(estimate_eigenvalues(h, prm->cheb_eig_iterations, &h->eig_min, &h->eig_max));
    h->eig_valid = true;
  }
  if (use_mg) {
    TRY(mg_build(h, prm));
    TRY(mg_setup(h, prm, picard));
  }
  h->mixed_ready = true;
  return MPDG_OK;
}

static int cg_chebyshev(mpdg_heat *h, const mpdg_solver_params *prm, double *x, const double *b,
                        mpdg_solve_stats *stats)
{
  const int64_t N = h->n_dofs;
  const bool use_mg = prm->preconditioner == MPDG_PRECOND_MG_F32;
  const bool picard = prm->cheb_picard && h->law == MPDG_LAW_LINEAR_K && h->tab.conductivity_q;
  if (!h->mixed_ready) TRY(mixed_prepare(h, prm));
  h->mixed_ready = false;
  double bmax = prm->cheb_max_factor * h->eig_max;
  double amin = std::max(h->eig_min, prm->cheb_min_fraction * bmax);
  double theta = 0.5 * (bmax + amin), delta = 0.5 * (bmax - amin);
  const int k = prm->cheb_degree;
  std::vector<float> c1, c2;
  cheb_coefficients(theta, delta, k, c1, c2);
  if (use_mg) {
    theta = h->mg[0].theta;
    bmax = theta + h->mg[0].delta;
    amin = theta - h->mg[0].delta;
  }
  const float inv_theta = (float)(1.0 / theta);
  const int g = vgrid(h, N);
  TRY(enable_cell_rows(h, picard));
  const CellRows xr = cell_rows_of(h);
  int total_it = 0, restarts = 0;
  double res0 = -1.0, true_res = 0.0;
  int graph_state = 0;  // 0 not recorded yet, 1 replaying, -1 direct launches
  set_level_streams(h, h->stream);
  if (any_faces(h)) TRY(dvec(h, &h->face_dot, 1));
  for (;;) {
    TRY(initial_Ax(h, x));
    (xr.rows ? k_cgm_init<true> : k_cgm_init<false>)<<<g, VT, 0, h->stream>>>(
      N, b, h->r, h->Ap, h->r32, h->x32, h->d32, h->Ax32,
                                        h->inv_diag_f, inv_theta, h->st, h->partials, h->counter,
                                        prm->rel_tolerance, prm->abs_tolerance,
                                        res0 > 0.0 && prm->tol_reference_norm <= 0.0
                                          ? res0
                                          : prm->tol_reference_norm,
                                        prm->max_iterations - total_it, xr); ++h->launches;
    CU(cudaGetLastError());
    TRY(poll(h));
    if (res0 < 0.0) res0 = h->st_host->res0;
    auto precondition = [&]() -> int {
      if (use_mg) {
        TRY(mg_vcycle(h, picard));
        k_cgm_update_p<<<g, VT, 0, h->stream>>>(N, h->z, h->pv, h->Ap, h->st); ++h->launches;
        CU(cudaGetLastError());
        return MPDG_OK;
      }
      for (int j = 1; j <= k; ++j) {
        TRY(op_apply_f(h, h->Ax32, h->x32, h->st, picard, xr.rows));
        if (j < k) {
          (xr.rows ? k_cheb_step<true> : k_cheb_step<false>)<<<g, VT, 0, h->stream>>>(
            N, h->r32, h->x32, h->d32, h->Ax32, h->inv_diag_f,
                                               c1[j], c2[j], h->st, xr);
        } else {
          (xr.rows ? k_cheb_last<true> : k_cheb_last<false>)<<<g, VT, 0, h->stream>>>(
            N, h->r32, h->x32, h->d32, h->Ax32, h->inv_diag_f,
                                               c1[j], c2[j], h->r, h->Ap, h->z, h->st,
                                               h->partials, h->counter, xr);
        }
        ++h->launches;
      }
      k_cgm_update_p<<<g, VT, 0, h->stream>>>(N, h->z, h->pv, h->Ap, h->st); ++h->launches;
      CU(cudaGetLastError());
      return MPDG_OK;
    };
    if (!h->st_host->done) TRY(precondition());
    auto iteration = [&]() -> int {
      TRY(op_apply_d(h, h->Ap, h->pv, FIN_CG_ALPHA, nullptr, h->st));
      (xr.rows ? k_cgm_update_xr<true> : k_cgm_update_xr<false>)<<<g, VT, 0, h->stream>>>(
        N, x, h->r, h->pv, h->Ap, h->r32, h->x32, h->d32,
                                               h->inv_diag_f, inv_theta, h->st, h->partials,
                                               h->counter, xr); ++h->launches;
      TRY(precondition());
      return MPDG_OK;
    };
    // the first preconditioner call above has made every allocation an iteration needs
    if (graph_state == 0 && !h->st_host->done)
      graph_state = (graphs_enabled() && !h->timing && record_body(h, iteration)) ? 1 : -1;
    // iterations are issued in chunks between host polls of the device-side state; the kernels
    // of an iteration issued after convergence return at once, but each launch still costs a
    // few microseconds (~0.3 ms for the ~130 launches of a multigrid iteration, more than a
    // poll), so the first chunk is the previous solve's count (one less with multigrid) and
    // the next ones single iterations (without a count yet: 2, 4, 8, 16)
    int &hint = h->its_hint[use_mg ? 0 : 1];
    int chunk = hint > 0 ? std::max(1, use_mg ? hint - 1 : hint) : 2;
    while (!h->st_host->done) {
      for (int c = 0; c < chunk; ++c) {
        if (graph_state == 1) {
          CU(cudaGraphLaunch(h->body_exec, h->stream));
          h->launches += h->body_launches;
          h->vm64 += h->body_vm64;
          h->vm32 += h->body_vm32;
        } else {
          TRY(iteration());
        }
      }
      TRY(poll(h));
      chunk = hint > 0 ? 1 : std::min(chunk * 2, 16);
    }
    if (h->st_host->done == 1 && restarts == 0) hint = h->st_host->it;
    total_it += h->st_host->it;
    const int done = h->st_host->done, status = h->st_host->status;
    const double tol = h->st_host->tol;
    if (h->early_host && h->early_T && done == 1 && restarts == 0) {
      // the step's new T (T_g + x, Dirichlet values set, as the step forms it after the
      // solve), sent to the host now so that the download overlaps the recheck
      TRY(dvec(h, &h->t_out, N));
      k_sum<<<g, VT, 0, h->stream>>>(N, h->t_out, h->early_T, x); ++h->launches;
      TRY(distribute(h, h->t_out));
      CU(cudaEventRecord(h->ev_early, h->stream));
      CU(cudaStreamWaitEvent(h->copy_stream, h->ev_early, 0));
      CU(cudaMemcpyAsync(h->early_host, h->t_out, sizeof(double) * N, cudaMemcpyDeviceToHost,
                         h->copy_stream));
      h->early_sent = true;
    }
    // true residual recheck in FP64
    CU(zero_async(h, h->Ap, sizeof(double) * N, h->stream));
    TRY(op_apply_d(h, h->Ap, x, FIN_NONE, nullptr, nullptr));
    TRY(dvec(h, &h->w3, N));
    CU(cudaMemcpyAsync(h->w3, b, sizeof(double) * N, cudaMemcpyDeviceToDevice, h->stream));
    k_axpy<<<g, VT, 0, h->stream>>>(N, h->w3, -1.0, h->Ap); ++h->launches;
    double rr = 0.0;
    TRY(norms(h, h->w3, nullptr, &rr, nullptr));
    true_res = std::sqrt(rr);
    if (done == 1 && true_res > tol && total_it < prm->max_iterations && restarts < 5) {
      ++restarts;
      h->early_sent = false;  // the increment changes: the step downloads T itself
      continue;
    }
    if (stats) {
      stats->iterations = total_it;
      stats->status = (done == 1 && true_res <= tol * 1.0000001) ? MPDG_OK
                      : (done == 1 ? MPDG_ERR_NOT_CONVERGED : status);
      stats->initial_residual = res0;
      stats->final_residual = h->st_host->res;
      stats->true_residual = true_res;
      stats->lambda_min = amin;
      stats->lambda_max = bmax;
    }
    return MPDG_OK;
  }
}

// ---------------------------------------------------------------------------
// GMRES(m) with right preconditioning (deal.II SolverGMRES as LinearSolver::solve
// configures it, linear_solver.hpp:113-118): the monitored quantity is the
// unpreconditioned residual |b - A x|, estimated by the Givens-rotated
// least-squares residual. Arnoldi with classical Gram-Schmidt applied twice
// (one multi-dot and one multi-axpy pass per round); the small Hessenberg
// problem is solved on the host.
// ---------------------------------------------------------------------------
// cheb: flexible GMRES whose preconditioner is the FP32 Chebyshev-Jacobi polynomial of the
// FP32 operator (D unused); each preconditioned direction z_j is kept in FP32 and the FP64
// operator is applied to its exact FP64 widening, so x += Z y uses exactly the vectors the
// Arnoldi process saw
static int gmres(mpdg_heat *h, const mpdg_solver_params *prm, double *x, const double *b,
                 const double *D, mpdg_solve_stats *stats, bool cheb = false)
{
  const int64_t N = h->n_dofs;
  const int m = std::max(1, std::min(prm->gmres_restart > 0 ? prm->gmres_restart : 28,
                                     kMaxBasis - 1));
  if (h->gV && h->gV_m < m) return fail(MPDG_ERR_INVALID_ARGUMENT, "GMRES restart grew");
  if (!h->gV) {
    TRY(dvec(h, &h->gV, (int64_t)(m + 1) * N));
    h->gV_m = m;
  }
  std::vector<float> c1, c2;
  float inv_theta = 1.f;
  const int kdeg = prm->cheb_degree;
  if (cheb) {
    if (kdeg < 1) return fail(MPDG_ERR_INVALID_ARGUMENT, "cheb_degree < 1");
    if (h->gZ && h->gZ_m < m) return fail(MPDG_ERR_INVALID_ARGUMENT, "GMRES restart grew");
    if (!h->gZ) {
      TRY(dvec(h, &h->gZ, (int64_t)m * N));
      h->gZ_m = m;
    }
    if (!h->st_run) {
      TRY(dvec(h, &h->st_run, 1));
      CU(zero_async(h, h->st_run, sizeof(SolverState), h->stream));  // done = 0, forever
    }
    TRY(ensure_workspace_f32(h));
    TRY(refresh_f32(h));
    if (h->diag_f_dirty) {
      k_cast_f<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->inv_diag, h->inv_diag_f); ++h->launches;
      CU(cudaGetLastError());
      h->diag_f_dirty = false;
    }
    if (!h->eig_valid || !prm->cheb_eig_reuse) {
      TRY(estimate_eigenvalues(h, prm->cheb_eig_iterations, &h->eig_min, &h->eig_max));
      h->eig_valid = true;
    }
    const double bmax = prm->cheb_max_factor * h->eig_max;
    const double amin = std::max(h->eig_min, prm->cheb_min_fraction * bmax);
    const double theta = 0.5 * (bmax + amin), delta = 0.5 * (bmax - amin);
    cheb_coefficients(theta, delta, kdeg, c1, c2);
    inv_theta = (float)(1.0 / theta);
  }
  // z = P(v_j): Chebyshev steps of the FP32 operator from v_j, stored in Z_j, widened into z
  auto precondition = [&](const double *vj, int j) -> int {
    float *zj = h->gZ + (int64_t)j * N;
    const int gg32 = vgrid(h, N);
    k_fgm_cheb_start<<<gg32, VT, 0, h->stream>>>(N, vj, h->r32, zj, h->d32, h->Ax32,
                                                 h->inv_diag_f, inv_theta);
    ++h->launches;
    for (int s = 1; s <= kdeg; ++s) {
      TRY(op_apply_f(h, h->Ax32, zj, nullptr, false));
      k_cheb_step<false><<<gg32, VT, 0, h->stream>>>(N, h->r32, zj, h->d32, h->Ax32, h->inv_diag_f,
                                              c1[s], c2[s], h->st_run, CellRows());
      ++h->launches;
    }
    k_widen<<<gg32, VT, 0, h->stream>>>(N, zj, h->z);
    ++h->launches;
    CU(cudaGetLastError());
    return MPDG_OK;
  };
  TRY(dvec(h, &h->gsmall, 4 * kMaxBasis));
  TRY(ensure_workspace(h));
  TRY(dvec(h, &h->z, N));
  double *V = h->gV, *hcol = h->gsmall, *ydev = h->gsmall + kMaxBasis;
  const int g = std::min(vgrid(h, N), h->sm_count * 4);
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), gg(m + 1), y(m), hc(kMaxBasis);
  double *hhost = h->scal_host;  // pinned, >= 8 doubles; larger reads go through hc below
  (void)hhost;
  int it = 0, status = MPDG_ERR_NOT_CONVERGED;
  double tol = 0.0, res = 0.0, res0 = -1.0;
  auto host_read = [&](const double *dev, double *dst, int cnt) -> int {
    TRY(read_to_host(h, h->rd_map, dev, sizeof(double) * cnt));  // cnt <= m <= kMaxBasis
    memcpy(dst, h->rd_host, sizeof(double) * cnt);
    return MPDG_OK;
  };
  for (;;) {
    TRY(initial_Ax(h, x));
    k_residual<<<g, VT, 0, h->stream>>>(N, b, h->Ap, V);
    ++h->launches;
    double rr = 0.0;
    TRY(norms(h, V, nullptr, &rr, nullptr));
    const double beta = std::sqrt(rr);
    if (res0 < 0.0) {
      res0 = beta;
      tol = std::max(prm->abs_tolerance,
                     prm->rel_tolerance * (prm->tol_reference_norm > 0.0 ? prm->tol_reference_norm : beta));
    }
    res = beta;
    if (!std::isfinite(beta)) {
      status = MPDG_ERR_NAN;
      break;
    }
    if (beta <= tol) {
      status = MPDG_OK;
      break;
    }
    if (it >= prm->max_iterations) break;
    k_scale_precond<<<g, VT, 0, h->stream>>>(N, V, 1.0 / beta, D, h->z);
    ++h->launches;
    if (cheb) TRY(precondition(V, 0));
    std::fill(gg.begin(), gg.end(), 0.0);
    std::fill(H.begin(), H.end(), 0.0);
    gg[0] = beta;
    int jj = 0;
    bool stop = false;
    for (int j = 0; j < m; ++j) {
      double *w = V + (int64_t)(j + 1) * N;
      CU(zero_async(h, w, sizeof(double) * N, h->stream));
      TRY(op_apply_d(h, w, h->z, FIN_NONE, nullptr, nullptr));
      for (int pass = 0; pass < 2; ++pass) {
        k_multidot<<<g, VT, 0, h->stream>>>(N, V, N, j + 1, w, h->partials, h->counter, hcol);
        k_multi_axpy<<<g, VT, 0, h->stream>>>(N, V, N, j + 1, hcol, w);
        h->launches += 2;
        TRY(host_read(hcol, hc.data(), j + 1));
        for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] += hc[i];
      }
      double ww = 0.0;
      TRY(norms(h, w, nullptr, &ww, nullptr));
      const double hn = std::sqrt(ww);
      H[(size_t)(j + 1) * m + j] = hn;
      for (int i = 0; i < j; ++i) {
        const double a = H[(size_t)i * m + j], c = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * c;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * c;
      }
      const double a = H[(size_t)j * m + j], c = H[(size_t)(j + 1) * m + j];
      const double r = std::sqrt(a * a + c * c);
      cs[j] = r > 0.0 ? a / r : 1.0;
      sn[j] = r > 0.0 ? c / r : 0.0;
      H[(size_t)j * m + j] = r;
      H[(size_t)(j + 1) * m + j] = 0.0;
      gg[j + 1] = -sn[j] * gg[j];
      gg[j] = cs[j] * gg[j];
      ++it;
      jj = j + 1;
      res = std::fabs(gg[j + 1]);
      if (!std::isfinite(res)) {
        status = MPDG_ERR_NAN;
        stop = true;
        break;
      }
      if (res <= tol || it >= prm->max_iterations || hn == 0.0) break;
      k_scale_precond<<<g, VT, 0, h->stream>>>(N, w, 1.0 / hn, D, h->z);
      ++h->launches;
      // the cycle's last direction is not preconditioned (Z holds m vectors; a restart
      // begins from the new residual)
      if (cheb && j + 1 < m) TRY(precondition(w, j + 1));
    }
    if (stop) break;
    // y = R^-1 g, x += M^-1 V y
    for (int i = jj - 1; i >= 0; --i) {
      double sacc = gg[i];
      for (int k = i + 1; k < jj; ++k) sacc -= H[(size_t)i * m + k] * y[k];
      y[i] = sacc / H[(size_t)i * m + i];
    }
    CU(cudaMemcpyAsync(ydev, y.data(), sizeof(double) * jj, cudaMemcpyHostToDevice, h->stream));
    if (cheb)
      k_fgmres_update<<<g, VT, 0, h->stream>>>(N, h->gZ, N, jj, ydev, x);
    else
      k_gmres_update<<<g, VT, 0, h->stream>>>(N, V, N, jj, ydev, D, x);
    ++h->launches;
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(h->stream));  // y lives on the host stack
    if (res <= tol) {
      status = MPDG_OK;
      break;
    }
    if (it >= prm->max_iterations) break;
  }
  if (stats) {
    stats->iterations = it;
    stats->status = status;
    stats->initial_residual = res0;
    stats->final_residual = res;
    stats->true_residual = res;
  }
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" void mpdg_solver_params_default(mpdg_solver_params *p)
{
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->solver = MPDG_SOLVER_CG;
  p->preconditioner = MPDG_PRECOND_JACOBI;
  p->max_iterations = 10000;
  p->rel_tolerance = 1e-12;
  p->abs_tolerance = 1e-20;
  p->gmres_restart = 28;
  p->cheb_degree = 4;
  p->cheb_eig_iterations = 12;
  p->cheb_max_factor = 1.2;
  p->cheb_min_fraction = 0.0;
  p->tol_reference_norm = 0.0;
  p->mg_smoothing_degree = 2;
  p->mg_coarse_degree = 8;
  p->mg_smoothing_range = 8.0;
  p->mg_min_cells = 4;
  p->mg_fine_pre_steps = -1;
  p->mg_fine_post_steps = -1;
}

extern "C" void mpdg_step_params_default(mpdg_step_params *p)
{
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->newton_max_iterations = 10;
  p->newton_residual_tolerance = 1e-9;
  p->newton_correction_tolerance = 1e-10;
  p->predictor = MPDG_PREDICTOR_LINEAR;
  p->single_linearization = 0;
  mpdg_solver_params_default(&p->linear);
}

static void release(mpdg_heat *h)
{
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->copy_stream) {
    cudaStreamSynchronize(h->copy_stream);
    cudaStreamDestroy(h->copy_stream);
    cudaEventDestroy(h->ev_source);
    cudaEventDestroy(h->ev_commit);
    cudaEventDestroy(h->ev_inputs);
    cudaEventDestroy(h->ev_early);
    for (int k = 0; k < mpdg_heat::kMaxSlabs; ++k) cudaEventDestroy(h->ev_slab[k]);
    h->copy_stream = nullptr;
  }
  for (MGLevel &lv : h->mg)
    if (lv.own && lv.h) {
      release(lv.h);
      delete lv.h;
    }
  h->mg.clear();
  if (h->body_exec) cudaGraphExecDestroy(h->body_exec);
  h->body_exec = nullptr;
  if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
  h->cap_stream = nullptr;
  drain_events(h);
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  h->ev_pool.clear();
  for (void *p : h->owned) cudaFree(p);
  h->owned.clear();
  if (h->st_host) cudaFreeHost(h->st_host);
  if (h->scal_host) cudaFreeHost(h->scal_host);
  if (h->rd_host) cudaFreeHost(h->rd_host);
  if (h->tc_err_host) cudaFreeHost(h->tc_err_host);
  h->tc_err_host = nullptr;
  h->st_host = nullptr;
  h->scal_host = nullptr;
  h->rd_host = nullptr;
}

// vertices of the box mesh: interior vertices perturbed by a counter hash of
// (seed, 3 * vertex + component), uniform in +-perturb * h
static std::vector<double> box_vertices(const mpdg_mesh_desc &desc)
{
  const int64_t nv = (int64_t)(desc.cells[0] + 1) * (desc.cells[1] + 1) * (desc.cells[2] + 1);
  std::vector<double> vert(3 * nv);
  double hc[3];
  for (int e = 0; e < 3; ++e) hc[e] = (desc.hi[e] - desc.lo[e]) / desc.cells[e];
  for (int c = 0; c <= desc.cells[2]; ++c)
    for (int b = 0; b <= desc.cells[1]; ++b)
      for (int a = 0; a <= desc.cells[0]; ++a) {
        const int idx[3] = {a, b, c};
        const int64_t v = a + (int64_t)(desc.cells[0] + 1) * (b + (int64_t)(desc.cells[1] + 1) * c);
        bool interior = true;
        for (int e = 0; e < 3; ++e)
          if (idx[e] == 0 || idx[e] == desc.cells[e]) interior = false;
        for (int e = 0; e < 3; ++e) {
          double x = desc.lo[e] + hc[e] * idx[e];
          if (interior) {
            uint64_t r = desc.seed * 0xD1B54A32D192ED03ULL + (uint64_t)(3 * v + e);
            r += 0x9E3779B97F4A7C15ULL;
            r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ULL;
            r = (r ^ (r >> 27)) * 0x94D049BB133111EBULL;
            r ^= r >> 31;
            const double u = 2.0 * ((double)(r >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
            x += desc.perturb * hc[e] * u;
          }
          vert[3 * v + e] = x;
        }
      }
  return vert;
}

// verts: host vertices of a deformed mesh ((cells + 1)^3 x 3), or null to generate them
static int create_impl(const mpdg_mesh_desc *desc, int device, const std::vector<double> *verts,
                       mpdg_heat **out);

extern "C" int mpdg_heat_create(const mpdg_mesh_desc *desc, int device, mpdg_heat **out)
{
  return create_impl(desc, device, nullptr, out);
}

extern "C" int mpdg_heat_create_slab(const mpdg_mesh_desc *global, int z_begin, int z_end,
                                     int device, mpdg_heat **out)
{
  if (!global || !out) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (z_begin < 0 || z_end > global->cells[2] || z_end <= z_begin || global->cells[0] < 1 ||
      global->cells[1] < 1)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "slab range outside the mesh");
  mpdg_mesh_desc d = *global;
  d.cells[2] = z_end - z_begin;
  const double hz = (global->hi[2] - global->lo[2]) / global->cells[2];
  d.lo[2] = global->lo[2] + hz * z_begin;
  d.hi[2] = z_end == global->cells[2] ? global->hi[2] : global->lo[2] + hz * z_end;
  if (z_begin > 0) d.dirichlet_mask &= ~16;
  if (z_end < global->cells[2]) d.dirichlet_mask &= ~32;
  if (!(global->perturb > 0.0)) return create_impl(&d, device, nullptr, out);
  // the global mesh's vertex planes z_begin .. z_end
  const std::vector<double> all = box_vertices(*global);
  const int64_t plane = (int64_t)(global->cells[0] + 1) * (global->cells[1] + 1);
  std::vector<double> verts(all.begin() + 3 * plane * z_begin,
                            all.begin() + 3 * plane * (z_end + 1));
  return create_impl(&d, device, &verts, out);
}

static int create_impl(const mpdg_mesh_desc *desc, int device, const std::vector<double> *verts,
                       mpdg_heat **out)
{
  if (!desc || !out) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (desc->degree < 1 || desc->degree > 6)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "degree must be in 1..6");
  for (int e = 0; e < 3; ++e) {
    if (desc->cells[e] < 1) return fail(MPDG_ERR_INVALID_ARGUMENT, "cells must be >= 1");
    if (!(desc->hi[e] > desc->lo[e])) return fail(MPDG_ERR_INVALID_ARGUMENT, "empty box");
  }
  if (desc->perturb < 0.0 || desc->perturb >= 0.5)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "perturb must be in [0, 0.5)");
  const int64_t nd0 = (int64_t)desc->degree * desc->cells[0] + 1,
                nd1 = (int64_t)desc->degree * desc->cells[1] + 1,
                nd2 = (int64_t)desc->degree * desc->cells[2] + 1;
  if (nd0 > (1 << 30) || nd1 > (1 << 30) || nd2 > (1 << 30))
    return fail(MPDG_ERR_INVALID_ARGUMENT, "mesh too large");
  CU(cudaSetDevice(device));
  mpdg_heat *h = new mpdg_heat();
  h->device = device;
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
  h->desc = *desc;
  h->p = desc->degree;
  h->n = h->p + 1;
  h->npt = h->n * h->n * h->n;
  for (int e = 0; e < 3; ++e) {
    h->dims.m[e] = desc->cells[e];
    h->dims.nd[e] = h->p * desc->cells[e] + 1;
    h->hcell[e] = (desc->hi[e] - desc->lo[e]) / desc->cells[e];
  }
  h->dims.p = h->p;
  h->dims.dmask = desc->dirichlet_mask & 63;
  h->n_dofs = nd0 * nd1 * nd2;
  h->n_cells = (int64_t)desc->cells[0] * desc->cells[1] * desc->cells[2];
  h->geo = desc->perturb > 0.0 ? 1 : 0;
  h->tab = table_for(h->n);
  int rc = upload_tables(device, h->n);
  if (rc != MPDG_OK) {
    delete h;
    return rc;
  }
  auto cleanup = [&](int code) {
    release(h);
    delete h;
    return code;
  };
  if ((rc = dalloc(h, (void **)&h->partials, sizeof(double) * 4 * kPartialsPerValue)) != MPDG_OK)
    return cleanup(rc);
  if ((rc = dalloc(h, (void **)&h->counter, sizeof(unsigned) * 4)) != MPDG_OK) return cleanup(rc);
  if ((rc = dalloc(h, (void **)&h->st, sizeof(SolverState))) != MPDG_OK) return cleanup(rc);
  if ((rc = dalloc(h, (void **)&h->scal, sizeof(double) * 8)) != MPDG_OK) return cleanup(rc);
  if (cudaHostAlloc((void **)&h->st_host, sizeof(SolverState), cudaHostAllocMapped) !=
          cudaSuccess ||
      cudaHostAlloc((void **)&h->scal_host, sizeof(double) * 8, cudaHostAllocMapped) !=
          cudaSuccess ||
      cudaHostAlloc((void **)&h->rd_host, sizeof(double) * kMaxBasis, cudaHostAllocMapped) !=
          cudaSuccess)
    return cleanup(fail(MPDG_ERR_OUT_OF_MEMORY, "cudaHostAlloc"));
  if (cudaHostGetDevicePointer((void **)&h->st_map, h->st_host, 0) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&h->scal_map, h->scal_host, 0) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&h->rd_map, h->rd_host, 0) != cudaSuccess)
    return cleanup(fail(MPDG_ERR_CUDA, "cudaHostGetDevicePointer"));
  cudaMemset(h->counter, 0, sizeof(unsigned) * 4);
  cudaMemset(h->st, 0, sizeof(SolverState));
  memset(h->st_host, 0, sizeof(SolverState));
  if (h->geo == 1) {
    // vertices on the host (counter-hash perturbation of interior vertices), then
    // per-quadrature-point geometry on the device
    const int64_t nv = (int64_t)(desc->cells[0] + 1) * (desc->cells[1] + 1) * (desc->cells[2] + 1);
    std::vector<double> gen;
    if (!verts) gen = box_vertices(*desc);
    const std::vector<double> &vert = verts ? *verts : gen;
    if ((int64_t)vert.size() != 3 * nv) return cleanup(fail(MPDG_ERR_INVALID_ARGUMENT, "vertex count"));
    if ((rc = dvec(h, &h->vert, 3 * nv)) != MPDG_OK) return cleanup(rc);
    if ((rc = dvec(h, &h->geoq, h->n_cells * 7 * h->npt)) != MPDG_OK) return cleanup(rc);
    if (cudaMemcpy(h->vert, vert.data(), sizeof(double) * 3 * nv, cudaMemcpyHostToDevice) !=
        cudaSuccess)
      return cleanup(fail(MPDG_ERR_CUDA, "vertex upload"));
    const Tables1D t1 = make_tables(h->n);
    Q1D q1;
    for (int i = 0; i < h->n; ++i) {
      q1.xg[i] = t1.xg[i];
      q1.wg[i] = t1.wg[i];
      q1.xl[i] = t1.xl[i];
    }
    const int64_t total = h->n_cells * h->npt;
    k_geometry<<<vgrid(h, total), VT>>>(h->n_cells, h->dims, h->n, q1, h->vert, h->geoq);
    if (cudaDeviceSynchronize() != cudaSuccess) return cleanup(fail(MPDG_ERR_CUDA, "geometry"));
  }
  mpdg_material m0;
  memset(&m0, 0, sizeof(m0));
  m0.law = MPDG_LAW_CONSTANT;
  m0.rho_l = m0.cp_l = m0.k_l = 1.0;
  m0.rho_s = m0.cp_s = m0.k_s = 1.0;
  m0.rho_g = m0.cp_g = m0.k_g = 1.0;
  m0.T_liquidus = 1.0;
  h->mat = m0;
  *out = h;
  return MPDG_OK;
}

extern "C" int mpdg_heat_destroy(mpdg_heat *h)
{
  if (!h) return MPDG_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  release(h);
  delete h;
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_stream(mpdg_heat *h, void *stream)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  h->stream = (cudaStream_t)stream;
  return MPDG_OK;
}

extern "C" int mpdg_heat_n_dofs(const mpdg_heat *h, int64_t *n)
{
  if (!h || !n) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  *n = h->n_dofs;
  return MPDG_OK;
}

extern "C" int mpdg_heat_n_cells(const mpdg_heat *h, int64_t *n)
{
  if (!h || !n) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  *n = h->n_cells;
  return MPDG_OK;
}

extern "C" int mpdg_heat_dof_dims(const mpdg_heat *h, int dims[3])
{
  if (!h || !dims) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  for (int e = 0; e < 3; ++e) dims[e] = h->dims.nd[e];
  return MPDG_OK;
}

extern "C" int mpdg_heat_device_bytes(const mpdg_heat *h, int64_t *bytes)
{
  if (!h || !bytes) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  *bytes = h->bytes;
  return MPDG_OK;
}

// d(rho_cp)/dT (T_lin - T_old) / dt enters the tangent when rho*cp depends on T
static void set_need_told(mpdg_heat *h)
{
  const mpdg_material *m = &h->mat;
  h->need_told = 0;
  if (m->law == MPDG_LAW_LIQUID_SOLID || m->law == MPDG_LAW_GAS_LIQUID_SOLID)
    h->need_told = m->volume_specific
                     ? (m->rho_l * m->cp_l != m->rho_s * m->cp_s)
                     : (m->rho_l != m->rho_s || m->cp_l != m->cp_s || h->latent > 0.0);
}

extern "C" int mpdg_heat_set_material(mpdg_heat *h, const mpdg_material *m)
{
  if (!h || !m) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (m->law < 0 || m->law > 4) return fail(MPDG_ERR_INVALID_ARGUMENT, "unknown material law");
  if (h->vel && m->law == MPDG_LAW_LINEAR_K)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "a velocity field is not available with the linear-k law");
  if ((m->law == MPDG_LAW_LIQUID_SOLID || m->law == MPDG_LAW_GAS_LIQUID_SOLID) && !m->sharp &&
      !(m->T_liquidus > m->T_solidus))
    return fail(MPDG_ERR_INVALID_ARGUMENT, "liquidus must exceed solidus");
  if (h->latent > 0.0 && m->volume_specific)
    return fail(MPDG_ERR_NOT_SUPPORTED,
                "the apparent capacity (latent heat) is not implemented for the volume specific "
                "heat capacity");
  h->mat = *m;
  h->law = m->law;
  set_need_told(h);
  h->diag_valid = false;
  h->eig_valid = false;
  h->cf_dirty = true;
  h->tf_dirty = true;
  h->tk_dirty = true;
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_latent_heat(mpdg_heat *h, double latent_heat, int profile)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  if (!(latent_heat >= 0.0) || !std::isfinite(latent_heat) || profile < MPDG_APPARENT_QLQ ||
      profile > MPDG_APPARENT_POLY4_BELL)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "latent heat >= 0 and a known apparent-capacity profile");
  if (latent_heat > 0.0 && h->mat.volume_specific)
    return fail(MPDG_ERR_NOT_SUPPORTED,
                "the apparent capacity (latent heat) is not implemented for the volume specific "
                "heat capacity");
  h->latent = latent_heat;
  h->acap = profile;
  set_need_told(h);
  h->diag_valid = false;
  h->eig_valid = false;
  h->cf_dirty = true;
  h->tf_dirty = true;
  h->tk_dirty = true;
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_dirichlet_values(mpdg_heat *h, const double values[6])
{
  if (!h || !values) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  for (int f = 0; f < 6; ++f)
    if (!std::isfinite(values[f])) return fail(MPDG_ERR_INVALID_ARGUMENT, "Dirichlet value not finite");
  for (int f = 0; f < 6; ++f) h->desc.dirichlet_value[f] = values[f];
  return MPDG_OK;
}

extern "C" int mpdg_material_eval(const mpdg_material *m, double latent_heat, int profile,
                                  double T, double H, double out[4])
{
  if (!m || !out) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (profile < MPDG_APPARENT_QLQ || profile > MPDG_APPARENT_POLY4_BELL || !(latent_heat >= 0.0))
    return fail(MPDG_ERR_INVALID_ARGUMENT, "latent heat >= 0 and a known apparent-capacity profile");
  MatParams<double> p;
  memset(&p, 0, sizeof(p));
  p.rho_l = m->rho_l, p.cp_l = m->cp_l, p.k_l = m->k_l;
  p.rho_s = m->rho_s, p.cp_s = m->cp_s, p.k_s = m->k_s;
  p.rho_g = m->rho_g, p.cp_g = m->cp_g, p.k_g = m->k_g;
  p.T_liq = m->T_liquidus, p.T_sol = m->T_solidus, p.k1 = m->k1;
  p.inv_mushy = m->T_liquidus != m->T_solidus ? 1.0 / (m->T_liquidus - m->T_solidus) : 0.0;
  p.sharp = m->sharp;
  p.vs = m->volume_specific;
  p.latent = latent_heat;
  p.acap = profile;
  if (latent_heat > 0.0 && m->volume_specific)
    return fail(MPDG_ERR_NOT_SUPPORTED, "apparent capacity with the volume specific capacity");
  switch (m->law) {
    case MPDG_LAW_CONSTANT: mat_eval<0>(p, T, out[0], out[1], out[2], out[3]); break;
    case MPDG_LAW_LINEAR_K: mat_eval<1>(p, T, out[0], out[1], out[2], out[3]); break;
    case MPDG_LAW_LIQUID_SOLID: mat_eval<2>(p, T, out[0], out[1], out[2], out[3]); break;
    case MPDG_LAW_GAS_LIQUID_SOLID: {
      const double w = m->sharp_gas_liquid ? (H > 0.5 ? 1.0 : 0.0) : H;
      mat_eval_w(p, T, w, out[0], out[1], out[2], out[3]);
      break;
    }
    default: return fail(MPDG_ERR_NOT_SUPPORTED, "host evaluation: laws 0, 1, 2 and 4");
  }
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_fields(mpdg_heat *h, const double *heaviside, const double *velocity)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  if (velocity && h->law == MPDG_LAW_LINEAR_K)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "a velocity field is not available with the linear-k law");
  h->Hf = heaviside;
  h->vel = velocity;
  h->cf_dirty = true;
  h->tf_dirty = true;
  h->tk_dirty = true;
  h->diag_valid = false;
  h->eig_valid = false;
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_boundary(mpdg_heat *h, int face, int type, double h_conv,
                                      double T_inf_conv, double emissivity, double T_inf_rad,
                                      double q_n)
{
  if (!h || face < 0 || face > 5 || type < 0 || type > 7)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "bad boundary face or type");
  if ((type & MPDG_BC_NEUMANN) && (type & (MPDG_BC_CONVECTION | MPDG_BC_RADIATION)))
    return fail(MPDG_ERR_INVALID_ARGUMENT,
                "It is not allowed to specify both Neumann and radiation and/or convection "
                "boundary conditions at the same face.");
  if ((type & MPDG_BC_CONVECTION | type & MPDG_BC_RADIATION | type & MPDG_BC_NEUMANN) &&
      (h->dims.dmask & (1 << face)))
    return fail(MPDG_ERR_INVALID_ARGUMENT, "face carries Dirichlet constraints");
  h->btype[face] = type;
  h->bh[face] = h_conv;
  h->bTc[face] = T_inf_conv;
  h->beps[face] = emissivity;
  h->bTr[face] = T_inf_rad;
  h->bqn[face] = q_n;
  h->lin_f_dirty = true;
  h->tf_dirty = true;
  h->tk_dirty = true;
  h->diag_valid = false;
  h->eig_valid = false;
  return MPDG_OK;
}

extern "C" int mpdg_heat_reset_time_increment(mpdg_heat *h, double dt)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  if (dt != h->dt) h->tf_dirty = true;
  h->dt = dt;
  h->eig_valid = false;
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_linearization(mpdg_heat *h, const double *T, const double *T_old)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  h->T_lin = T;
  h->T_old = T_old;
  h->lin_f_dirty = true;
  h->tf_dirty = true;
  h->tk_dirty = true;
  return MPDG_OK;
}

extern "C" int mpdg_heat_vmult(mpdg_heat *h, double *dst, const double *src)
{
  if (!h || !dst || !src) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  CU(zero_async(h, dst, sizeof(double) * h->n_dofs, h->stream));
  return op_apply_d(h, dst, src, FIN_NONE, nullptr, nullptr);
}

extern "C" int mpdg_heat_vmult_f32(mpdg_heat *h, float *dst, const float *src)
{
  if (!h || !dst || !src) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  CU(zero_async(h, dst, sizeof(float) * h->n_dofs, h->stream));
  return op_apply_f(h, dst, src, nullptr);
}

extern "C" int mpdg_heat_vmult_f32_picard(mpdg_heat *h, float *dst, const float *src)
{
  if (!h || !dst || !src) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (h->law != MPDG_LAW_LINEAR_K || !h->tab.conductivity_q)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "Picard operator: linear-k law, degree <= 4 only");
  CU(cudaSetDevice(h->device));
  TRY(ensure_lin(h));
  TRY(dvec(h, &h->kq, h->n_cells * h->npt));
  CellArgs<double> a = cell_args<double>(h);
  a.Tl = h->T_lin;
  CU(h->tab.conductivity_q(a, h->kq, h->law, h->stream, h->sm_count));
  ++h->launches;
  CU(zero_async(h, dst, sizeof(float) * h->n_dofs, h->stream));
  return op_apply_f(h, dst, src, nullptr, true);
}

__global__ void k_to_cell_rows(int64_t N, CellRows c, const float *__restrict__ lex)
{
  GRID_STRIDE(i, N) cell_rows_store(c, i, lex[i]);
}

extern "C" int mpdg_heat_cell_rows_size(const mpdg_heat *h, int64_t *n_floats)
{
  if (!h || !n_floats) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (h->p != 3) return fail(MPDG_ERR_NOT_SUPPORTED, "cell rows: FE_Q(3) only");
  *n_floats = cell_rows_size(h);
  return MPDG_OK;
}

extern "C" int mpdg_heat_to_cell_rows_f32(mpdg_heat *h, float *rows, const float *lex)
{
  if (!h || !rows || !lex) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (h->p != 3) return fail(MPDG_ERR_NOT_SUPPORTED, "cell rows: FE_Q(3) only");
  if (h->n_dofs >= ((int64_t)1 << 32)) return fail(MPDG_ERR_NOT_SUPPORTED, "cell rows: >= 2^32 DoFs");
  CU(cudaSetDevice(h->device));
  CellRows c;
  c.rows = rows;
  c.nd0 = (unsigned)h->dims.nd[0];
  c.rs = 4u * (unsigned)h->dims.m[0];
  k_to_cell_rows<<<vgrid(h, h->n_dofs), VT, 0, h->stream>>>(h->n_dofs, c, lex);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_vmult_f32_picard_rows(mpdg_heat *h, float *dst, const float *src_rows)
{
  if (!h || !dst || !src_rows) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (h->law != MPDG_LAW_LINEAR_K || !h->tab.conductivity_q)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "Picard operator: linear-k law, degree <= 4 only");
  if (h->p != 3 || !h->tab.vmult_picard_rows)
    return fail(MPDG_ERR_NOT_SUPPORTED, "cell rows: FE_Q(3) only");
  CU(cudaSetDevice(h->device));
  TRY(ensure_lin(h));
  TRY(dvec(h, &h->kq, h->n_cells * h->npt));
  CellArgs<double> a = cell_args<double>(h);
  a.Tl = h->T_lin;
  CU(h->tab.conductivity_q(a, h->kq, h->law, h->stream, h->sm_count));
  ++h->launches;
  CU(zero_async(h, dst, sizeof(float) * h->n_dofs, h->stream));
  return op_apply_f(h, dst, nullptr, nullptr, true, src_rows);
}

extern "C" int mpdg_heat_picard_cell_rows(const mpdg_heat *h) { return h && h->rows_on ? 1 : 0; }

extern "C" int mpdg_heat_set_picard_tensor_cores(mpdg_heat *h, int on)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  h->picard_tc = on ? 1 : 0;
  h->eig_valid = false;
  return MPDG_OK;
}

extern "C" int mpdg_picard_tc_matrices(float *out)
{
  if (!out) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  optc::build_gmat(out);
  return MPDG_OK;
}

extern "C" int mpdg_heat_picard_tensor_cores(const mpdg_heat *h)
{
  return h && picard_tc_on(h) ? 1 : 0;
}

extern "C" int mpdg_heat_inverse_diagonal_f32_picard(mpdg_heat *h, float *inv_diag)
{
  if (!h || !inv_diag) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (h->law != MPDG_LAW_LINEAR_K || !h->tab.conductivity_q)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "Picard operator: linear-k law, degree <= 4 only");
  CU(cudaSetDevice(h->device));
  TRY(ensure_lin(h));
  TRY(dvec(h, &h->kq, h->n_cells * h->npt));
  CellArgs<double> a = cell_args<double>(h);
  a.Tl = h->T_lin;
  CU(h->tab.conductivity_q(a, h->kq, h->law, h->stream, h->sm_count));
  ++h->launches;
  TRY(picard_inverse_diagonal(h));
  h->diag_f_dirty = true;  // inv_diag_f now holds the Picard diagonal
  CU(cudaMemcpyAsync(inv_diag, h->inv_diag_f, sizeof(float) * h->n_dofs,
                     cudaMemcpyDeviceToDevice, h->stream));
  return MPDG_OK;
}

static int compute_diag(mpdg_heat *h, double *d, bool invert)
{
  TRY(ensure_dt(h));
  TRY(ensure_lin(h));
  TRY(ensure_fields(h));
  CU(zero_async(h, d, sizeof(double) * h->n_dofs, h->stream));
  CellArgs<double> a = cell_args<double>(h);
  a.g.q = h->geoq;
  a.cf = h->cf;
  a.dst = d;
  a.Tl = h->T_lin;
  a.To = h->T_old;
  CU(h->tab.diag(a, h->geo, klaw(h), h->stream, h->sm_count));
  ++h->launches;
  if (any_faces(h)) TRY(launch_faces<double>(h, 2, d, nullptr, h->T_lin, nullptr, nullptr));
  if (!invert) {
    CU(cudaGetLastError());
    return MPDG_OK;
  }
  k_invert_diag<<<vgrid(h, h->n_dofs), VT, 0, h->stream>>>(h->n_dofs, d); ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_compute_inverse_diagonal(mpdg_heat *h, double *inv_diag)
{
  if (!h || !inv_diag) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  return compute_diag(h, inv_diag);
}

extern "C" int mpdg_heat_compute_diagonal(mpdg_heat *h, double *diag)
{
  if (!h || !diag) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  return compute_diag(h, diag, false);
}

static int create_rhs(mpdg_heat *h, double *dst, const double *src, const double *q)
{
  TRY(ensure_dt(h));
  if (!h->T_lin) return fail(MPDG_ERR_INVALID_ARGUMENT, "create_rhs needs set_linearization");
  TRY(ensure_lin(h));
  TRY(ensure_fields(h));
  CellArgs<double> a = cell_args<double>(h);
  a.g.q = h->geoq;
  a.cf = h->cf;
  a.dst = dst;
  a.Tl = h->T_lin;
  a.To = src;
  a.qs = q;
  if (!q && h->source.on) a.source = h->source;
  CU(h->tab.rhs(a, h->geo, klaw(h), h->stream, h->sm_count));
  ++h->launches;
  if (any_faces(h)) TRY(launch_faces<double>(h, 1, dst, nullptr, h->T_lin, nullptr, nullptr));
  return MPDG_OK;
}

// create_rhs with the nodal source arriving in z-slabs on the copy stream (upload_source): the
// cells of layers [slab_cz[k], slab_cz[k + 1]) are applied as a sub-box of the mesh (base
// pointers at its first node plane, per-cell fields at its first cell, the z faces Dirichlet only
// where they are the mesh's) once slab k has arrived; the nodes shared by two sub-boxes receive
// both contributions through the atomic scatter, as from neighbouring cells of one launch
static int create_rhs_slabs(mpdg_heat *h, double *dst, const double *src, const double *q)
{
  TRY(ensure_dt(h));
  if (!h->T_lin) return fail(MPDG_ERR_INVALID_ARGUMENT, "create_rhs needs set_linearization");
  TRY(ensure_lin(h));
  TRY(ensure_fields(h));
  CellArgs<double> a = cell_args<double>(h);
  const MeshDims d = a.d;
  const int64_t layer_cells = (int64_t)d.m[0] * d.m[1];
  const int64_t plane = (int64_t)d.nd[0] * d.nd[1];
  for (int k = 0; k < h->n_slabs; ++k) {
    const int cz0 = h->slab_cz[k], cz1 = h->slab_cz[k + 1];
    CU(cudaStreamWaitEvent(h->stream, h->ev_slab[k], 0));
    if (cz1 <= cz0) continue;
    CellArgs<double> b = a;
    const int64_t c0 = (int64_t)cz0 * layer_cells, n0 = (int64_t)d.p * cz0 * plane;
    b.n_cells = (int64_t)(cz1 - cz0) * layer_cells;
    b.d.m[2] = cz1 - cz0;
    b.d.nd[2] = d.p * (cz1 - cz0) + 1;
    if (cz0 > 0) b.d.dmask &= ~16;
    if (cz1 < d.m[2]) b.d.dmask &= ~32;
    b.g.q = h->geoq ? h->geoq + c0 * 7 * h->npt : nullptr;
    b.cf = h->cf ? h->cf + c0 * 5 * h->npt : nullptr;
    b.dst = dst + n0;
    b.Tl = h->T_lin + n0;
    b.To = src + n0;
    b.qs = q + n0;
    CU(h->tab.rhs(b, h->geo, klaw(h), h->stream, h->sm_count));
    ++h->launches;
  }
  if (any_faces(h)) TRY(launch_faces<double>(h, 1, dst, nullptr, h->T_lin, nullptr, nullptr));
  return MPDG_OK;
}

// the host source into host_q on the copy stream in z-slabs of node planes (slab k holds the
// planes up to p slab_cz[k + 1], so it completes every cell of layers below slab_cz[k + 1]),
// ev_slab[k] after each and ev_source after the last
static int upload_source(mpdg_heat *h, const double *host_src)
{
  const MeshDims &d = h->dims;
  const int K = std::max(1, std::min(mpdg_heat::kMaxSlabs, d.m[2]));
  const int64_t plane = (int64_t)d.nd[0] * d.nd[1];
  int64_t pl0 = 0;
  for (int k = 0; k <= K; ++k) h->slab_cz[k] = (int)(((int64_t)k * d.m[2]) / K);
  for (int k = 0; k < K; ++k) {
    const int64_t pl1 = k + 1 < K ? (int64_t)d.p * h->slab_cz[k + 1] + 1 : d.nd[2];
    CU(cudaMemcpyAsync(h->host_q + pl0 * plane, host_src + pl0 * plane,
                       sizeof(double) * (size_t)((pl1 - pl0) * plane), cudaMemcpyHostToDevice,
                       h->copy_stream));
    CU(cudaEventRecord(h->ev_slab[k], h->copy_stream));
    pl0 = pl1;
  }
  CU(cudaEventRecord(h->ev_source, h->copy_stream));
  h->n_slabs = K;
  return MPDG_OK;
}

extern "C" int mpdg_heat_create_rhs(mpdg_heat *h, double *dst, const double *src,
                                    const double *heat_source)
{
  if (!h || !dst || !src) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  return create_rhs(h, dst, src, heat_source);
}

// ---------------------------------------------------------------------------
// host-vector verbs (OperatorMatrixFree's VectorType is the host vector
// LinearAlgebra::distributed::Vector<number>, operator_base.hpp:192): the vectors are
// copied into device mirrors the handle keeps, renumbered from the caller's DoF order to
// the lexicographic one on the device, and the results copied back
// ---------------------------------------------------------------------------
__global__ void k_perm_in(int64_t N, const int64_t *__restrict__ lex, const double *__restrict__ x,
                          double *__restrict__ y)
{
  GRID_STRIDE(i, N) y[lex[i]] = x[i];
}

__global__ void k_perm_out(int64_t N, const int64_t *__restrict__ lex, const double *__restrict__ y,
                           double *__restrict__ x)
{
  GRID_STRIDE(i, N) x[i] = y[lex[i]];
}

static int host_mirrors(mpdg_heat *h)
{
  TRY(dvec(h, &h->hv_a, h->n_dofs));
  TRY(dvec(h, &h->hv_b, h->n_dofs));
  TRY(dvec(h, &h->hv_c, h->n_dofs));
  return MPDG_OK;
}

// host vector in caller numbering -> device vector in lexicographic numbering
static int upload_host(mpdg_heat *h, double *dev, const double *host)
{
  const int64_t N = h->n_dofs;
  if (!h->perm) {
    CU(cudaMemcpyAsync(dev, host, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream));
    return MPDG_OK;
  }
  CU(cudaMemcpyAsync(h->hv_c, host, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream));
  k_perm_in<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->perm, h->hv_c, dev);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

// device vector in lexicographic numbering -> host vector in caller numbering; synchronises
static int download_host(mpdg_heat *h, double *host, const double *dev)
{
  const int64_t N = h->n_dofs;
  const double *from = dev;
  if (h->perm) {
    k_perm_out<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->perm, dev, h->hv_c);
    ++h->launches;
    CU(cudaGetLastError());
    from = h->hv_c;
  }
  CU(cudaMemcpyAsync(host, from, sizeof(double) * N, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_dof_permutation(mpdg_heat *h, const int64_t *lex_of_dof)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  CU(cudaSetDevice(h->device));
  if (!lex_of_dof) {
    h->perm = nullptr;  // identity (the buffer stays owned by the handle)
    return MPDG_OK;
  }
  const int64_t N = h->n_dofs;
  std::vector<unsigned char> seen((size_t)N, 0);
  for (int64_t i = 0; i < N; ++i) {
    const int64_t v = lex_of_dof[i];
    if (v < 0 || v >= N || seen[(size_t)v])
      return fail(MPDG_ERR_INVALID_ARGUMENT,
                  "DoF permutation: entry " + std::to_string(i) + " is out of range or repeated");
    seen[(size_t)v] = 1;
  }
  TRY(dvec(h, &h->perm_buf, N));
  CU(cudaMemcpyAsync(h->perm_buf, lex_of_dof, sizeof(int64_t) * N, cudaMemcpyHostToDevice,
                     h->stream));
  CU(cudaStreamSynchronize(h->stream));
  h->perm = h->perm_buf;
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_linearization_host(mpdg_heat *h, const double *T, const double *T_old)
{
  if (!h || !T) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  TRY(host_mirrors(h));
  TRY(dvec(h, &h->hv_T, h->n_dofs));
  TRY(upload_host(h, h->hv_T, T));
  if (T_old) {
    TRY(dvec(h, &h->hv_To, h->n_dofs));
    TRY(upload_host(h, h->hv_To, T_old));
  }
  return mpdg_heat_set_linearization(h, h->hv_T, T_old ? h->hv_To : nullptr);
}

extern "C" int mpdg_heat_vmult_host(mpdg_heat *h, double *dst, const double *src)
{
  if (!h || !dst || !src) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  TRY(host_mirrors(h));
  TRY(upload_host(h, h->hv_a, src));
  TRY(mpdg_heat_vmult(h, h->hv_b, h->hv_a));
  return download_host(h, dst, h->hv_b);
}

extern "C" int mpdg_heat_compute_inverse_diagonal_host(mpdg_heat *h, double *inv_diag)
{
  if (!h || !inv_diag) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  TRY(host_mirrors(h));
  TRY(compute_diag(h, h->hv_b));
  return download_host(h, inv_diag, h->hv_b);
}

extern "C" int mpdg_heat_create_rhs_host(mpdg_heat *h, double *dst, const double *src,
                                         const double *heat_source)
{
  if (!h || !dst || !src) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  TRY(host_mirrors(h));
  TRY(upload_host(h, h->hv_b, dst));
  TRY(upload_host(h, h->hv_a, src));
  double *q = nullptr;
  if (heat_source) {
    TRY(dvec(h, &h->host_q, h->n_dofs));
    TRY(upload_host(h, h->host_q, heat_source));
    q = h->host_q;
  }
  TRY(create_rhs(h, h->hv_b, h->hv_a, q));
  return download_host(h, dst, h->hv_b);
}

static int distribute(mpdg_heat *h, double *u)
{
  DirArgs a;
  a.d = h->dims;
  for (int f = 0; f < 6; ++f) a.val[f] = h->desc.dirichlet_value[f];
  for (int f = 0; f < 6; ++f) {
    if (!(h->dims.dmask & (1 << f))) continue;
    const int dir = f / 2;
    const int e1 = dir == 0 ? 1 : 0, e2 = dir == 2 ? 1 : 2;
    const int64_t cnt = (int64_t)h->dims.nd[e1] * h->dims.nd[e2];
    k_distribute<<<vgrid(h, cnt), VT, 0, h->stream>>>(a, f, u); ++h->launches;
  }
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_distribute_constraints(mpdg_heat *h, double *u)
{
  if (!h || !u) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  return distribute(h, u);
}

extern "C" int mpdg_heat_l2_norm(mpdg_heat *h, const double *u, double *norm)
{
  if (!h || !u || !norm) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  CellArgs<double> a = cell_args<double>(h);
  a.g.q = h->geoq;
  a.src = u;
  a.out = h->scal;
  CU(h->tab.norm(a, h->geo, 0, h->stream, h->sm_count));
  ++h->launches;
  TRY(read_to_host(h, h->scal_map, h->scal, sizeof(double)));
  *norm = std::sqrt(h->scal_host[0]);
  return MPDG_OK;
}

static PosArgs pos_args(const mpdg_heat *h)
{
  PosArgs a;
  a.d = h->dims;
  a.geo = h->geo;
  for (int e = 0; e < 3; ++e) {
    a.lo[e] = h->desc.lo[e];
    a.hc[e] = h->hcell[e];
  }
  const Tables1D t1 = make_tables(h->n);
  for (int i = 0; i < h->n; ++i) {
    a.q1.xg[i] = t1.xg[i];
    a.q1.wg[i] = t1.wg[i];
    a.q1.xl[i] = t1.xl[i];
  }
  a.vert = h->vert;
  return a;
}

extern "C" int mpdg_heat_support_points(mpdg_heat *h, double *xyz)
{
  if (!h || !xyz) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  k_support_points<<<vgrid(h, h->n_dofs), VT, 0, h->stream>>>(h->n_dofs, pos_args(h), xyz); ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

static int laser_args(const mpdg_laser *laser, LaserArgs &g)
{
  const int pr = laser->profile;
  if (pr < MPDG_LASER_UNIFORM || pr > MPDG_LASER_GUSAROV)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "unknown laser intensity profile");
  memset(&g, 0, sizeof(g));
  g.profile = pr;
  g.planar = laser->planar != 0;
  g.power = laser->power;
  for (int e = 0; e < 3; ++e) {
    g.c[e] = laser->position[e];
    g.dir[e] = laser->direction[e];
  }
  g.radius = laser->radius;
  if (pr != MPDG_LASER_UNIFORM && !(g.radius > 0.0))
    return fail(MPDG_ERR_INVALID_ARGUMENT,
                "The laser beam radius must be greater than zero! Abort..");
  const double half_pi = 0.5 * M_PI;
  if (pr == MPDG_LASER_GAUSS_VOLUMETRIC) {
    const double s = g.radius * std::sqrt(half_pi);
    g.peak = g.power / (s * s * s);
  } else if (pr == MPDG_LASER_GAUSS_PROJECTION) {
    const double nrm = std::sqrt(g.dir[0] * g.dir[0] + g.dir[1] * g.dir[1] + g.dir[2] * g.dir[2]);
    if (!(std::fabs(nrm - 1.0) < 1e-8))
      return fail(MPDG_ERR_INVALID_ARGUMENT, "The line direction must be a unit vector");
    g.peak = g.power / (g.radius * g.radius * half_pi);
  } else if (pr == MPDG_LASER_GUSAROV) {
    g.rho = laser->reflectivity;
    g.beta = laser->extinction_coefficient;
    g.L = laser->layer_thickness;
    g.lambda = g.beta * g.L;
    g.a = std::sqrt(1.0 - g.rho);
    g.D = (1.0 - g.a) * (1.0 - g.a - g.rho * (1.0 + g.a)) * std::exp(-2.0 * g.a * g.lambda) -
          (1.0 + g.a) * (1.0 + g.a - g.rho * (1.0 - g.a)) * std::exp(2.0 * g.a * g.lambda);
  }
  return MPDG_OK;
}

extern "C" int mpdg_heat_laser_source(mpdg_heat *h, double *q, const mpdg_laser *laser)
{
  if (!h || !q || !laser) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  LaserArgs g;
  TRY(laser_args(laser, g));
  CU(cudaSetDevice(h->device));
  k_laser<<<vgrid(h, h->n_dofs), VT, 0, h->stream>>>(h->n_dofs, pos_args(h), g, q);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_laser(mpdg_heat *h, const mpdg_laser *laser)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  if (!laser) {
    h->source.on = 0;
    return MPDG_OK;
  }
  LaserArgs g;
  TRY(laser_args(laser, g));
  h->source.laser = g;
  h->source.pos = pos_args(h);
  h->source.on = 1;
  return MPDG_OK;
}

extern "C" int mpdg_heat_gaussian_source(mpdg_heat *h, double *q, double amplitude,
                                         const double center[3], double radius)
{
  if (!h || !q || !center || !(radius > 0.0)) return fail(MPDG_ERR_INVALID_ARGUMENT, "bad argument");
  CU(cudaSetDevice(h->device));
  k_gaussian<<<vgrid(h, h->n_dofs), VT, 0, h->stream>>>(h->n_dofs, pos_args(h), q, amplitude,
                                                        center[0], center[1], center[2],
                                                        1.0 / (radius * radius)); ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_preconditioner_update(mpdg_heat *h)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  CU(cudaSetDevice(h->device));
  TRY(dvec(h, &h->inv_diag, h->n_dofs));
  TRY(compute_diag(h, h->inv_diag));
  h->diag_valid = true;
  h->diag_f_dirty = true;
  h->eig_valid = false;
  return MPDG_OK;
}

extern "C" int mpdg_heat_preconditioner_vmult(mpdg_heat *h, double *dst, const double *src)
{
  if (!h || !dst || !src) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (!h->diag_valid) return fail(MPDG_ERR_INVALID_ARGUMENT, "preconditioner not updated");
  CU(cudaSetDevice(h->device));
  k_scale<<<vgrid(h, h->n_dofs), VT, 0, h->stream>>>(h->n_dofs, dst, src, h->inv_diag); ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

static int linear_solve(mpdg_heat *h, const mpdg_solver_params *prm, double *x, const double *b,
                        mpdg_solve_stats *stats)
{
  mpdg_solve_stats local;
  memset(&local, 0, sizeof(local));
  if (prm->solver == MPDG_SOLVER_GMRES) {
    if (prm->preconditioner == MPDG_PRECOND_MG_F32)
      return fail(MPDG_ERR_NOT_SUPPORTED,
                  "GMRES supports identity, Jacobi or FP32 Chebyshev-Jacobi preconditioning");
    const bool cheb = prm->preconditioner == MPDG_PRECOND_CHEBYSHEV_JACOBI_F32;
    const double *D = nullptr;
    if (prm->preconditioner == MPDG_PRECOND_JACOBI || cheb) {
      if (!h->diag_valid) return fail(MPDG_ERR_INVALID_ARGUMENT, "preconditioner not updated");
      if (!cheb) D = h->inv_diag;
    }
    TRY(gmres(h, prm, x, b, D, &local, cheb));
  } else if (prm->solver != MPDG_SOLVER_CG) {
    return fail(MPDG_ERR_INVALID_ARGUMENT, "unknown solver type");
  } else if (prm->preconditioner == MPDG_PRECOND_CHEBYSHEV_JACOBI_F32 ||
             prm->preconditioner == MPDG_PRECOND_MG_F32) {
    TRY(cg_chebyshev(h, prm, x, b, &local));
  } else {
    const double *D = nullptr;
    if (prm->preconditioner == MPDG_PRECOND_JACOBI) {
      if (!h->diag_valid) return fail(MPDG_ERR_INVALID_ARGUMENT, "preconditioner not updated");
      D = h->inv_diag;
    }
    TRY(cg_jacobi(h, prm, x, b, D, 0, &local));
  }
  if (stats) *stats = local;
  if (local.status != MPDG_OK)
    return fail(local.status, local.status == MPDG_ERR_NOT_CONVERGED
                                ? "linear solver did not converge"
                                : (local.status == MPDG_ERR_NAN ? "residual is not finite"
                                                                : "solver breakdown"));
  return MPDG_OK;
}

extern "C" int mpdg_heat_linear_solve(mpdg_heat *h, const mpdg_solver_params *prm, double *x,
                                      const double *b, mpdg_solve_stats *stats)
{
  if (!h || !prm || !x || !b) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  return linear_solve(h, prm, x, b, stats);
}

extern "C" int mpdg_heat_set_direction(mpdg_heat *h, const double *direction)
{
  if (!h || !direction) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  h->direction = direction;
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_guess(mpdg_heat *h, const double *guess)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  h->guess = guess;
  return MPDG_OK;
}

extern "C" int mpdg_heat_time_step(mpdg_heat *h, const mpdg_step_params *prm, double dt,
                                   double dt_old, double *T_cur, double *T_old,
                                   const double *heat_source, mpdg_step_stats *stats)
{
  if (!h || !prm || !T_cur || !T_old) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (prm->predictor == MPDG_PREDICTOR_GIVEN && !h->guess)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "predictor GIVEN needs mpdg_heat_set_guess");
  const bool with_direction = prm->predictor == MPDG_PREDICTOR_LINEAR_DIRECTION;
  if (with_direction && (!h->direction || !prm->single_linearization))
    return fail(MPDG_ERR_INVALID_ARGUMENT,
                "predictor LINEAR_DIRECTION needs mpdg_heat_set_direction and single_linearization");
  const int predictor = with_direction ? MPDG_PREDICTOR_LINEAR : prm->predictor;
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  const size_t vb = sizeof(double) * N;
  TRY(dvec(h, &h->w1, N));
  TRY(dvec(h, &h->w2, N));
  TRY(dvec(h, &h->z, N));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  CU(cudaEventRecord(e0, h->stream));
  mpdg_step_stats s;
  memset(&s, 0, sizeof(s));
  int rc = MPDG_OK;
  h->mixed_ready = false;
  do {
    // the Chebyshev / multigrid interval: kept across steps with cheb_eig_reuse until dt (or
    // the material or the mesh) changes; a solve that does not use it leaves it alone
    const bool uses_interval = prm->linear.preconditioner == MPDG_PRECOND_CHEBYSHEV_JACOBI_F32 ||
                               prm->linear.preconditioner == MPDG_PRECOND_MG_F32;
    if (h->dt != dt || (uses_interval && !prm->linear.cheb_eig_reuse)) h->eig_valid = false;
    h->dt = dt;
    // init_time_advance: predictor into w1, commit history, constraints
    if (h->rotate) {
      // the predicted T replaces T_{n-1} in its buffer and the two buffers swap roles
      if (predictor == MPDG_PREDICTOR_LINEAR && std::fabs(dt_old) >= 1e-12) {
        k_predict_inplace<<<vgrid(h, N), VT, 0, h->stream>>>(N, T_cur, T_old, dt / dt_old);
        ++h->launches;
      } else {
        const double *from = predictor == MPDG_PREDICTOR_GIVEN ? h->guess : T_cur;
        if ((rc = (cudaMemcpyAsync(T_old, from, vb, cudaMemcpyDeviceToDevice, h->stream) ==
                   cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, "predictor copy"))) != MPDG_OK)
          break;
      }
      std::swap(T_cur, T_old);
      h->rotated = true;
    } else if (predictor == MPDG_PREDICTOR_LINEAR && std::fabs(dt_old) >= 1e-12) {
      k_predict<<<vgrid(h, N), VT, 0, h->stream>>>(N, T_cur, T_old, h->w1, dt / dt_old); ++h->launches;
    } else if (predictor == MPDG_PREDICTOR_GIVEN) {
      if ((rc = (cudaMemcpyAsync(h->w1, h->guess, vb, cudaMemcpyDeviceToDevice, h->stream) ==
                 cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, "guess copy"))) != MPDG_OK) break;
    } else {
      if ((rc = (cudaMemcpyAsync(h->w1, T_cur, vb, cudaMemcpyDeviceToDevice, h->stream) ==
                 cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, "copy"))) != MPDG_OK) break;
    }
    if (!h->rotate) {
      cudaMemcpyAsync(T_old, T_cur, vb, cudaMemcpyDeviceToDevice, h->stream);
      cudaMemcpyAsync(T_cur, h->w1, vb, cudaMemcpyDeviceToDevice, h->stream);
    }
    if (h->record_commit) {
      // T_old is final here: its copy to the host runs on the copy stream during the step
      cudaEventRecord(h->ev_commit, h->stream);
      cudaStreamWaitEvent(h->copy_stream, h->ev_commit, 0);
      cudaMemcpyAsync(h->told_host, T_old, vb, cudaMemcpyDeviceToHost, h->copy_stream);
    }
    if ((rc = distribute(h, T_cur)) != MPDG_OK) break;
    h->T_lin = T_cur;
    h->T_old = T_old;
    h->lin_f_dirty = true;
    h->tf_dirty = true;
    h->tk_dirty = true;
    // JacobiPreconditioner::update; the multigrid preconditioner on the Picard operator
    // needs the FP64 diagonal only for a new Lanczos estimate
    const bool mg_picard = prm->linear.preconditioner == MPDG_PRECOND_MG_F32 &&
                           prm->linear.cheb_picard && h->law == MPDG_LAW_LINEAR_K &&
                           h->tab.conductivity_q;
    if (prm->linear.preconditioner != MPDG_PRECOND_IDENTITY &&
        (!mg_picard || !h->eig_valid || !prm->linear.cheb_eig_reuse)) {
      if ((rc = dvec(h, &h->inv_diag, N)) != MPDG_OK) break;
      if ((rc = compute_diag(h, h->inv_diag)) != MPDG_OK) break;
      h->diag_valid = true;
      h->diag_f_dirty = true;
    } else if (mg_picard) {
      h->diag_valid = false;  // the stored diagonal belongs to an earlier linearisation
    }
    if (prm->single_linearization) {
      // b = J T_g - R(T_g); solve J delta = -R(T_g) to |b - J T| <= tol |b|
      // J T_g first: it does not need the source, whose upload may still be running
      zero_async(h, h->z, vb, h->stream);
      if ((rc = op_apply_d(h, h->z, T_cur, FIN_NONE, nullptr, nullptr)) != MPDG_OK) break;
      // so is the mixed-precision preconditioner's set-up (it depends on T_lin only), unless it
      // has to estimate the fine level's interval (its Lanczos CG uses z, which holds J T_g)
      if (h->wait_source && h->eig_valid && prm->linear.cheb_eig_reuse &&
          prm->linear.solver == MPDG_SOLVER_CG &&
          (prm->linear.preconditioner == MPDG_PRECOND_CHEBYSHEV_JACOBI_F32 ||
           prm->linear.preconditioner == MPDG_PRECOND_MG_F32) &&
          (rc = mixed_prepare(h, &prm->linear)) != MPDG_OK)
        break;
      zero_async(h, h->w2, vb, h->stream);
      if (h->wait_source && h->n_slabs > 0 && heat_source) {
        if ((rc = create_rhs_slabs(h, h->w2, T_old, heat_source)) != MPDG_OK) break;
      } else {
        if (h->wait_source) cudaStreamWaitEvent(h->stream, h->ev_source, 0);
        if ((rc = create_rhs(h, h->w2, T_old, heat_source)) != MPDG_OK) break;
      }
      double rr = 0.0, bb = 0.0;
      if ((rc = norms(h, h->w2, h->z, &rr, &bb)) != MPDG_OK) break;
      mpdg_solver_params lp = prm->linear;
      lp.tol_reference_norm = std::sqrt(bb);
      lp.abs_tolerance = std::max(lp.abs_tolerance, 0.0);
      mpdg_solve_stats ls;
      memset(&ls, 0, sizeof(ls));
      if (with_direction) {
        // the increment solve starts from alpha d, alpha = argmin |r - alpha J d| (never a
        // larger initial residual than from 0); J d is computed once and handed to the solver
        if ((rc = dvec(h, &h->w3, N)) != MPDG_OK) break;
        zero_async(h, h->w3, vb, h->stream);
        if ((rc = op_apply_d(h, h->w3, h->direction, FIN_NONE, nullptr, nullptr)) != MPDG_OK) break;
        double jj = 0.0, jr = 0.0;
        if ((rc = norms(h, h->w3, h->w2, &jj, &jr)) != MPDG_OK) break;
        const double rj = 0.5 * (jr - jj - rr);
        const double alpha = jj > 0.0 ? rj / jj : 0.0;
        k_scale_copy<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->w1, h->direction, alpha);
        ++h->launches;
        h->x_Ax = h->w3;
        h->x_Ax_scale = alpha;
        rr = std::max(rr - alpha * rj, 0.0);
      } else {
        zero_async(h, h->w1, vb, h->stream);
        h->x_zero = true;
      }
      h->early_T = h->early_host ? T_cur : nullptr;  // T_g, for the early download of T
      rc = linear_solve(h, &lp, h->w1, h->w2, &ls);
      h->early_T = nullptr;
      h->x_zero = false;
      h->x_Ax = nullptr;
      if (rc != MPDG_OK) break;
      k_axpy<<<vgrid(h, N), VT, 0, h->stream>>>(N, T_cur, 1.0, h->w1); ++h->launches;
      if ((rc = distribute(h, T_cur)) != MPDG_OK) break;
      s.linear_iterations = ls.iterations;
      s.newton_iterations = 1;
      s.converged = 1;
      s.initial_relative_residual = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
    } else {
      for (int i = 0; i < prm->newton_max_iterations; ++i) {
        zero_async(h, h->w2, vb, h->stream);
        if (h->wait_source) cudaStreamWaitEvent(h->stream, h->ev_source, 0);
        if ((rc = create_rhs(h, h->w2, T_old, heat_source)) != MPDG_OK) break;
        zero_async(h, h->w1, vb, h->stream);
        mpdg_solve_stats ls;
        memset(&ls, 0, sizeof(ls));
        h->x_zero = true;
        rc = linear_solve(h, &prm->linear, h->w1, h->w2, &ls);
        h->x_zero = false;
        if (rc != MPDG_OK) break;
        s.linear_iterations += ls.iterations;
        double rr = 0.0, dd = 0.0;
        if ((rc = norms(h, h->w2, nullptr, &rr, nullptr)) != MPDG_OK) break;
        if ((rc = norms(h, h->w1, nullptr, &dd, nullptr)) != MPDG_OK) break;
        if (std::sqrt(rr) < prm->newton_residual_tolerance &&
            std::sqrt(dd) < prm->newton_correction_tolerance) {
          s.converged = 1;
          break;
        }
        k_axpy<<<vgrid(h, N), VT, 0, h->stream>>>(N, T_cur, 1.0, h->w1); ++h->launches;
        if ((rc = distribute(h, T_cur)) != MPDG_OK) break;
        h->lin_f_dirty = true;
        h->tf_dirty = true;
        h->tk_dirty = true;
        s.newton_iterations = i + 1;
      }
      if (rc == MPDG_OK && !s.converged)
        rc = fail(MPDG_ERR_NEWTON_NOT_CONVERGED, "Newton-Raphson did not converge");
    }
  } while (0);
  h->mixed_ready = false;
  cudaEventRecord(e1, h->stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s.step_ms = ms;
  if (stats) *stats = s;
  if (rc == MPDG_OK) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MPDG_ERR_CUDA, cudaGetErrorString(e));
  }
  return rc;
}

static int ensure_copy_stream(mpdg_heat *h)
{
  if (!h->copy_stream) {
    CU(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    CU(cudaEventCreateWithFlags(&h->ev_source, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&h->ev_commit, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&h->ev_inputs, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&h->ev_early, cudaEventDisableTiming));
    for (int k = 0; k < mpdg_heat::kMaxSlabs; ++k)
      CU(cudaEventCreateWithFlags(&h->ev_slab[k], cudaEventDisableTiming));
  }
  return MPDG_OK;
}

extern "C" int mpdg_heat_time_step_host(mpdg_heat *h, const mpdg_step_params *prm, double dt,
                                        double dt_old, double *T_cur, double *T_old,
                                        const double *heat_source, mpdg_step_stats *stats)
{
  if (!h || !prm || !T_cur || !T_old) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  const size_t vb = sizeof(double) * N;
  TRY(dvec(h, &h->host_T, N));
  TRY(dvec(h, &h->host_To, N));
  if (heat_source) TRY(dvec(h, &h->host_q, N));
  TRY(ensure_copy_stream(h));
  // T and T_old are needed first (predictor, history commit); the source only by
  // create_rhs, so its copy runs on the copy stream while the step starts
  CU(cudaMemcpyAsync(h->host_T, T_cur, vb, cudaMemcpyHostToDevice, h->stream));
  CU(cudaMemcpyAsync(h->host_To, T_old, vb, cudaMemcpyHostToDevice, h->stream));
  CU(cudaEventRecord(h->ev_inputs, h->stream));
  if (heat_source) {
    CU(cudaStreamWaitEvent(h->copy_stream, h->ev_inputs, 0));  // one transfer at a time
    TRY(upload_source(h, heat_source));
  }
  // the new T_old (= the input T) is final once the step has committed the history: the
  // step starts its copy back then, so it runs while the solve computes; T follows at the end
  h->wait_source = heat_source != nullptr;
  h->record_commit = true;
  h->told_host = T_old;
  // with the mixed-precision CG the new T goes back during the solver's residual recheck
  // (copy stream; the T input was read from this buffer at the start of the call)
  h->early_host = T_cur;
  h->early_sent = false;
  const int rc = mpdg_heat_time_step(h, prm, dt, dt_old, h->host_T, h->host_To,
                                     heat_source ? h->host_q : nullptr, stats);
  h->early_host = nullptr;
  h->wait_source = false;
  h->n_slabs = 0;
  h->record_commit = false;
  h->told_host = nullptr;
  if (rc != MPDG_OK) {
    cudaStreamSynchronize(h->copy_stream);
    h->early_sent = false;
    return rc;
  }
  if (!h->early_sent) {
    // an early download invalidated by a restart still writes T_cur: let it finish first
    CU(cudaStreamSynchronize(h->copy_stream));
    CU(cudaMemcpyAsync(T_cur, h->host_T, vb, cudaMemcpyDeviceToHost, h->stream));
  }
  h->early_sent = false;
  CU(cudaStreamSynchronize(h->copy_stream));
  CU(cudaStreamSynchronize(h->stream));
  return MPDG_OK;
}

extern "C" int mpdg_heat_load_history(mpdg_heat *h, const double *T_host, const double *T_old_host)
{
  if (!h || !T_host || !T_old_host) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  TRY(dvec(h, &h->res_T, N));
  TRY(dvec(h, &h->res_To, N));
  CU(cudaMemcpyAsync(h->res_T, T_host, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream));
  CU(cudaMemcpyAsync(h->res_To, T_old_host, sizeof(double) * N, cudaMemcpyHostToDevice,
                     h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return MPDG_OK;
}

extern "C" int mpdg_heat_store_history(mpdg_heat *h, double *T_host, double *T_old_host)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  if (!h->res_T) return fail(MPDG_ERR_INVALID_ARGUMENT, "no resident history: call load_history");
  CU(cudaSetDevice(h->device));
  const size_t vb = sizeof(double) * h->n_dofs;
  if (T_host) CU(cudaMemcpyAsync(T_host, h->res_T, vb, cudaMemcpyDeviceToHost, h->stream));
  if (T_old_host) CU(cudaMemcpyAsync(T_old_host, h->res_To, vb, cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return MPDG_OK;
}

extern "C" int mpdg_heat_time_step_resident(mpdg_heat *h, const mpdg_step_params *prm, double dt,
                                            double dt_old, const double *heat_source,
                                            double *T_out, mpdg_step_stats *stats)
{
  if (!h || !prm) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (!h->res_T) return fail(MPDG_ERR_INVALID_ARGUMENT, "no resident history: call load_history");
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  const size_t vb = sizeof(double) * N;
  if (heat_source) {
    TRY(dvec(h, &h->host_q, N));
    TRY(ensure_copy_stream(h));
    // the source is first needed by create_rhs: its upload (in z-slabs, each applied by the
    // residual as it arrives) overlaps the predictor, the history commit, the first operator
    // application and the mixed-precision preconditioner's set-up (the previous source buffer
    // is free: every call ends synchronised)
    CU(cudaEventRecord(h->ev_inputs, h->stream));
    CU(cudaStreamWaitEvent(h->copy_stream, h->ev_inputs, 0));
    TRY(upload_source(h, heat_source));
  }
  // the two history buffers swap roles: the predictor overwrites T_{n-1} in place
  h->wait_source = heat_source != nullptr;
  h->rotate = true;
  h->rotated = false;
  // with the mixed-precision CG the new T is downloaded as soon as the increment has converged,
  // during the solver's FP64 residual recheck (on the copy stream)
  if (T_out) {
    TRY(ensure_copy_stream(h));
    h->early_host = T_out;
  }
  h->early_sent = false;
  const int rc = mpdg_heat_time_step(h, prm, dt, dt_old, h->res_T, h->res_To,
                                     heat_source ? h->host_q : nullptr, stats);
  h->early_host = nullptr;
  h->wait_source = false;
  h->n_slabs = 0;
  h->rotate = false;
  if (h->rotated) std::swap(h->res_T, h->res_To);
  h->rotated = false;
  if (rc != MPDG_OK) {
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    h->early_sent = false;
    return rc;
  }
  if (T_out && !h->early_sent) {
    // an early download invalidated by a restart still writes T_out: let it finish first
    if (h->copy_stream) CU(cudaStreamSynchronize(h->copy_stream));
    CU(cudaMemcpyAsync(T_out, h->res_T, vb, cudaMemcpyDeviceToHost, h->stream));
  }
  h->early_sent = false;
  if (h->copy_stream) CU(cudaStreamSynchronize(h->copy_stream));
  CU(cudaStreamSynchronize(h->stream));
  return MPDG_OK;
}

extern "C" int mpdg_heat_set_timing(mpdg_heat *h, int enable)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  h->timing = enable != 0;
  return MPDG_OK;
}

extern "C" int mpdg_heat_get_counters(mpdg_heat *h, mpdg_counters *c, int reset)
{
  if (!h || !c) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  CU(cudaStreamSynchronize(h->stream));
  drain_events(h);
  // this handle's launches and those of its multigrid levels
  c->launches = h->launches;
  c->vmult64_calls = h->vm64;
  c->vmult32_calls = h->vm32;
  for (MGLevel &lv : h->mg)
    if (lv.h && lv.h != h) {
      c->launches += lv.h->launches;
      c->vmult64_calls += lv.h->vm64;
      c->vmult32_calls += lv.h->vm32;
    }
  c->vmult64_ms = h->ms64;
  c->vmult32_ms = h->ms32;
  if (reset) {
    h->launches = h->vm64 = h->vm32 = 0;
    h->ms64 = h->ms32 = 0.0;
    for (MGLevel &lv : h->mg)
      if (lv.h && lv.h != h) lv.h->launches = lv.h->vm64 = lv.h->vm32 = 0;
  }
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// stages of a Jacobi-CG iteration split across ranks (z-slab decomposition)
//
// The caller owns the collectives: each stage reduces over this rank's owned DoFs (the first
// n_owned entries; a shared plane is owned by the upper slab) into device doubles, which the
// caller all-reduces (NCCL on device buffers) before the next stage; the step lengths alpha
// and beta are device scalars too, so an iteration needs no host round trip except the
// convergence test.
// ---------------------------------------------------------------------------
__global__ void k_dcg_start(int64_t N, int64_t n_owned, const double *__restrict__ b,
                            const double *__restrict__ Ax, const double *__restrict__ D,
                            double *r, double *z, double *p, double *partials,
                            unsigned *counter, double *out)
{
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(i, N)
  {
    const double ri = b[i] - (Ax ? Ax[i] : 0.0);
    const double zi = D[i] * ri;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    if (i < n_owned) {
      v[0] += ri * zi;
      v[1] += ri * ri;
    }
  }
  double tot[2];
  if (grid_sum<2>(v, partials, counter, tot)) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

__global__ void k_dcg_dot(int64_t n_owned, const double *__restrict__ a,
                          const double *__restrict__ b, double *partials, unsigned *counter,
                          double *out)
{
  double v[1] = {0.0};
  GRID_STRIDE(i, n_owned) v[0] += a[i] * b[i];
  double tot[1];
  if (grid_sum<1>(v, partials, counter, tot)) out[0] = tot[0];
}

// x += alpha p, r -= alpha Ap, z = D r; out = (r.z, r.r) over the owned DoFs
__global__ void k_dcg_update(int64_t N, int64_t n_owned, double *x, double *r, double *z,
                             const double *__restrict__ p, const double *__restrict__ Ap,
                             const double *__restrict__ D, const double *__restrict__ alpha,
                             double *partials, unsigned *counter, double *out)
{
  const double al = *alpha;
  double v[2] = {0.0, 0.0};
  GRID_STRIDE(i, N)
  {
    x[i] += al * p[i];
    const double ri = r[i] - al * Ap[i];
    const double zi = D[i] * ri;
    r[i] = ri;
    z[i] = zi;
    if (i < n_owned) {
      v[0] += ri * zi;
      v[1] += ri * ri;
    }
  }
  double tot[2];
  if (grid_sum<2>(v, partials, counter, tot)) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

__global__ void k_dcg_direction(int64_t N, double *p, const double *__restrict__ z,
                                const double *__restrict__ beta)
{
  const double be = *beta;
  GRID_STRIDE(i, N) p[i] = z[i] + be * p[i];
}

static int dcg_check(mpdg_heat *h, int64_t n_owned)
{
  if (n_owned < 0 || n_owned > h->n_dofs)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "n_owned must be in [0, n_dofs]");
  return MPDG_OK;
}

extern "C" int mpdg_heat_dcg_start(mpdg_heat *h, int64_t n_owned, const double *b, const double *Ax,
                                   const double *inv_diag, double *r, double *z, double *p,
                                   double *partial)
{
  if (!h || !b || !inv_diag || !r || !z || !p || !partial)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  TRY(dcg_check(h, n_owned));
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  k_dcg_start<<<vgrid(h, N), VT, 0, h->stream>>>(N, n_owned, b, Ax, inv_diag, r, z, p,
                                                 h->partials, h->counter, partial);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_dcg_dot(mpdg_heat *h, int64_t n_owned, const double *a, const double *b,
                                 double *partial)
{
  if (!h || !a || !b || !partial) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  TRY(dcg_check(h, n_owned));
  CU(cudaSetDevice(h->device));
  k_dcg_dot<<<vgrid(h, std::max<int64_t>(n_owned, 1)), VT, 0, h->stream>>>(
    n_owned, a, b, h->partials, h->counter, partial);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_dcg_update(mpdg_heat *h, int64_t n_owned, double *x, double *r,
                                    double *z, const double *p, const double *Ap,
                                    const double *inv_diag, const double *alpha, double *partial)
{
  if (!h || !x || !r || !z || !p || !Ap || !inv_diag || !alpha || !partial)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  TRY(dcg_check(h, n_owned));
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  k_dcg_update<<<vgrid(h, N), VT, 0, h->stream>>>(N, n_owned, x, r, z, p, Ap, inv_diag, alpha,
                                                  h->partials, h->counter, partial);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_dcg_direction(mpdg_heat *h, double *p, const double *z, const double *beta)
{
  if (!h || !p || !z || !beta) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  k_dcg_direction<<<vgrid(h, N), VT, 0, h->stream>>>(N, p, z, beta);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

extern "C" int mpdg_heat_invert_diagonal(mpdg_heat *h, double *d)
{
  if (!h || !d) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  k_invert_diag<<<vgrid(h, h->n_dofs), VT, 0, h->stream>>>(h->n_dofs, d);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// FE L2 norm that allocates nothing
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool, where raw driver allocations are forbidden or would
// break its accounting, and loops that must not pay the implicit device
// synchronisation of a first-use allocation. For them this variant of the L2
// norm keeps its reduction scratch (one partial sum per CTA plus the last-CTA
// election counter) in a fixed array in this file instead of handle memory,
// and writes the result to a device scalar the caller owns.
//
// Limits and sharing: the array holds kNoAllocSlots partial sums (128 KiB),
// i.e. the reduction grid may have at most kNoAllocSlots CTAs; a launch that
// would need more is rejected with MPDG_ERR_INVALID_ARGUMENT (it cannot happen
// on GPUs with up to 512 SMs). Every GPU that loads the library holds the
// array until the process exits. All calls on a device share it and it keeps
// the last call's contents; the counter is cleared at the start of each call,
// so calls that overlap on the GPU (different streams, or different host
// threads on one device) race and must be serialised by the caller. The first
// call on a device looks up the array's device address (cudaGetSymbolAddress)
// and caches it per device; that first call should come before any stream capture.
// The cached address is not valid after cudaDeviceReset on that device.
// ---------------------------------------------------------------------------
static constexpr int kNoAllocSlots = 16384;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots + 32];

static std::mutex g_noalloc_mutex;
static double *g_noalloc_addr[64];

__global__ void k_sqrt_scalar(double *x) { *x = sqrt(*x); }

// Device address of the static scratch array on `device` (the current device),
// looked up once per device on the first call there.
static int noalloc_scratch(int device, double **out)
{
  if (device < 0 || device >= 64) return fail(MPDG_ERR_INVALID_ARGUMENT, "device id");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[device]) {
    double *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(MPDG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_addr[device] = p;
  }
  *out = g_noalloc_addr[device];
  return MPDG_OK;
}

extern "C" int mpdg_heat_l2_norm_noalloc(mpdg_heat *h, const double *u, double *norm)
{
  if (!h || !u || !norm) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  CU(cudaSetDevice(h->device));
  double *scratch = nullptr;
  TRY(noalloc_scratch(h->device, &scratch));
  int max_ctas_per_sm = 32;
  cudaDeviceGetAttribute(&max_ctas_per_sm, cudaDevAttrMaxBlocksPerMultiprocessor, h->device);
  const int64_t batches = (h->n_cells + cells_per_block(h->n) - 1) / cells_per_block(h->n);
  const int64_t slots = std::min<int64_t>(batches, (int64_t)max_ctas_per_sm * h->sm_count);
  if (slots > kNoAllocSlots)
    return fail(MPDG_ERR_INVALID_ARGUMENT,
                "l2_norm_noalloc: the reduction needs " + std::to_string(slots) +
                  " partial sums, the static scratch holds " + std::to_string(kNoAllocSlots));
  unsigned *counter = reinterpret_cast<unsigned *>(scratch + kNoAllocSlots);
  CU(cudaMemsetAsync(counter, 0, sizeof(unsigned), h->stream));
  CellArgs<double> a = cell_args<double>(h);
  a.g.q = h->geoq;
  a.src = u;
  a.out = norm;
  a.partials = scratch;
  a.counter = counter;
  CU(h->tab.norm(a, h->geo, 0, h->stream, h->sm_count));
  k_sqrt_scalar<<<1, 1, 0, h->stream>>>(norm);
  CU(cudaGetLastError());
  h->launches += 2;
  return MPDG_OK;
}

// ---------------------------------------------------------------------------
// learned initial guess: sampling onto the network grid and prolongation back
// ---------------------------------------------------------------------------
// scale_sum (nullable, device): the increment scale is then sqrt(scale_sum[0] * inv_n) for
// s0 and s1, computed on the device (a zero scale gives zero features)
__global__ void k_learned_input(MeshDims d, int stride, int cx, int cy, int cz,
                                const double *__restrict__ T, const double *__restrict__ To,
                                const double *__restrict__ q, double dt, double s0, double s1,
                                double s2, const double *__restrict__ scale_sum, double inv_n,
                                float *in)
{
  const int64_t nc = (int64_t)cx * cy * cz;
  if (scale_sum) {
    s0 = s1 = sqrt(scale_sum[0] * inv_n);
    if (!(s0 > 0.0)) s0 = s1 = INFINITY;  // zero features
  }
  GRID_STRIDE(t, nc)
  {
    const int X = (int)(t % cx), Y = (int)((t / cx) % cy), Z = (int)(t / ((int64_t)cx * cy));
    const int64_t f = (int64_t)stride * X + (int64_t)d.nd[0] * ((int64_t)stride * Y + (int64_t)d.nd[1] * stride * Z);
    const double Tv = T[f];
    in[t] = (float)((Tv - To[f]) / s0);
    in[nc + t] = (float)(q ? dt * q[f] / s1 : 0.0);
    in[2 * nc + t] = (float)(Tv / s2);
  }
}

// trilinear prolongation of the sampled-grid field y to nodal DoF i
__device__ __forceinline__ double prolong_at(int64_t i, const MeshDims &d, int stride, int cx, int cy,
                                             int cz, const float *__restrict__ y)
{
  const int64_t I = i % d.nd[0], J = (i / d.nd[0]) % d.nd[1], K = i / ((int64_t)d.nd[0] * d.nd[1]);
  const int64_t pos[3] = {I, J, K};
  const int cdim[3] = {cx, cy, cz};
  int lo[3], hi[3];
  double w[3];
  for (int e = 0; e < 3; ++e) {
    lo[e] = (int)(pos[e] / stride);
    const int r = (int)(pos[e] - (int64_t)lo[e] * stride);
    hi[e] = lo[e] + (r > 0 ? 1 : 0);
    if (hi[e] >= cdim[e]) hi[e] = cdim[e] - 1;
    w[e] = (double)r / stride;
  }
  double s = 0.0;
  for (int c = 0; c < 8; ++c) {
    const int ix = (c & 1) ? hi[0] : lo[0], iy = (c & 2) ? hi[1] : lo[1], iz = (c & 4) ? hi[2] : lo[2];
    const double wt = ((c & 1) ? w[0] : 1.0 - w[0]) * ((c & 2) ? w[1] : 1.0 - w[1]) *
                      ((c & 4) ? w[2] : 1.0 - w[2]);
    if (wt != 0.0) s += wt * (double)y[ix + (int64_t)cx * (iy + (int64_t)cy * iz)];
  }
  return s;
}

__global__ void k_learned_guess(int64_t N, MeshDims d, int stride, int cx, int cy, int cz,
                                const double *__restrict__ T, const double *__restrict__ To,
                                const float *__restrict__ y, double s3, double *g)
{
  GRID_STRIDE(i, N) g[i] = 2.0 * T[i] - To[i] + s3 * prolong_at(i, d, stride, cx, cy, cz, y);
}

// the network's increment direction s3 P(y), zero at the Dirichlet DoFs
__global__ void k_learned_direction(int64_t N, MeshDims d, int stride, int cx, int cy, int cz,
                                    const float *__restrict__ y, double s3,
                                    const double *__restrict__ scale_sum, double inv_n, double *g)
{
  if (scale_sum) s3 = sqrt(scale_sum[0] * inv_n);
  GRID_STRIDE(i, N)
  {
    const int I = (int)(i % d.nd[0]), J = (int)((i / d.nd[0]) % d.nd[1]),
              K = (int)(i / ((int64_t)d.nd[0] * d.nd[1]));
    g[i] = constrained(d, I, J, K) ? 0.0 : s3 * prolong_at(i, d, stride, cx, cy, cz, y);
  }
}

// sum of (a - b)^2 into out[0] (last-CTA reduction)
__global__ void k_diff_sq(int64_t N, const double *__restrict__ a, const double *__restrict__ b,
                          double *partials, unsigned *counter, double *out)
{
  double v[1] = {0.0};
  GRID_STRIDE(i, N)
  {
    const double x = a[i] - b[i];
    v[0] += x * x;
  }
  double tot[1];
  if (grid_sum<1>(v, partials, counter, tot)) out[0] = tot[0];
}

static int learned_dims(mpdg_heat *h, int stride, int c[3])
{
  if (stride < 1) return fail(MPDG_ERR_INVALID_ARGUMENT, "stride must be >= 1");
  for (int e = 0; e < 3; ++e) {
    if ((h->dims.nd[e] - 1) % stride != 0)
      return fail(MPDG_ERR_INVALID_ARGUMENT, "(n_dofs per direction - 1) must be divisible by stride");
    c[e] = (h->dims.nd[e] - 1) / stride + 1;
  }
  return MPDG_OK;
}

extern "C" int mpdg_heat_learned_input(mpdg_heat *h, int stride, const double *T,
                                       const double *T_old, const double *heat_source, double dt,
                                       const double scales[3], float *input)
{
  if (!h || !T || !T_old || !scales || !input) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  int c[3];
  TRY(learned_dims(h, stride, c));
  CU(cudaSetDevice(h->device));
  const int64_t nc = (int64_t)c[0] * c[1] * c[2];
  k_learned_input<<<vgrid(h, nc), VT, 0, h->stream>>>(h->dims, stride, c[0], c[1], c[2], T, T_old,
                                                     heat_source, dt, scales[0], scales[1],
                                                     scales[2], nullptr, 0.0, input);
  CU(cudaGetLastError());
  ++h->launches;
  return MPDG_OK;
}

extern "C" int mpdg_unet_forward(mpdg_unet *u, const float *input, float *output);
extern "C" int mpdg_unet_set_stream(mpdg_unet *u, void *stream);
extern "C" int mpdg_unet_dims(const mpdg_unet *u, int dims[3]);

__global__ void k_lincomb(int64_t N, double *out, double a, const double *__restrict__ x, double b,
                          const double *__restrict__ y)
{
  GRID_STRIDE(i, N) out[i] = a * x[i] + b * (y ? y[i] : 0.0);
}

extern "C" int mpdg_heat_learned_guess(mpdg_heat *h, mpdg_unet *u, int stride, const double *T,
                                       const double *T_old, const double *heat_source, double dt,
                                       double T_scale, int line_search, double *guess,
                                       double *alpha_out)
{
  if (!h || !u || !T || !T_old || !guess) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (!(dt > 0.0) || !(T_scale > 0.0)) return fail(MPDG_ERR_INVALID_ARGUMENT, "dt and T_scale must be > 0");
  int c[3];
  TRY(learned_dims(h, stride, c));
  int ud[3];
  TRY(mpdg_unet_dims(u, ud));
  if (ud[0] != c[0] || ud[1] != c[1] || ud[2] != c[2])
    return fail(MPDG_ERR_INVALID_ARGUMENT,
                "network grid " + std::to_string(ud[0]) + "x" + std::to_string(ud[1]) + "x" +
                  std::to_string(ud[2]) + " does not match the sampled mesh grid " +
                  std::to_string(c[0]) + "x" + std::to_string(c[1]) + "x" + std::to_string(c[2]));
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  const int64_t nc = (int64_t)c[0] * c[1] * c[2];
  TRY(dalloc(h, reinterpret_cast<void **>(&h->nn_buf), sizeof(float) * 4 * nc));
  if (h->nn_buf_n == 0) h->nn_buf_n = nc;
  if (h->nn_buf_n != nc) return fail(MPDG_ERR_INVALID_ARGUMENT, "network grid changed");
  TRY(dvec(h, &h->w1, N));
  TRY(dvec(h, &h->w2, N));
  TRY(dvec(h, &h->w3, N));
  // per-sample scale: RMS of the time increment
  k_lincomb<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->w1, 1.0, T, -1.0, T_old);
  ++h->launches;
  double dd = 0.0;
  TRY(norms(h, h->w1, nullptr, &dd, nullptr));
  const double a = std::sqrt(dd / (double)N);
  // linear extrapolation 2 T - T_old (with Dirichlet values) into guess
  k_lincomb<<<vgrid(h, N), VT, 0, h->stream>>>(N, guess, 2.0, T, -1.0, T_old);
  ++h->launches;
  TRY(distribute(h, guess));
  if (!(a > 0.0)) {  // no history yet: the extrapolation is the guess
    if (alpha_out) *alpha_out = 0.0;
    return MPDG_OK;
  }
  const double scales[3] = {a, a, T_scale};
  TRY(mpdg_heat_learned_input(h, stride, T, T_old, heat_source, dt, scales, h->nn_buf));
  mpdg_unet_set_stream(u, h->stream);
  const int rc = mpdg_unet_forward(u, h->nn_buf, h->nn_buf + 3 * nc);
  if (rc != MPDG_OK) return fail(rc, "network forward failed");
  // d = a * P(y) (prolongated correction) into w1, zero at Dirichlet DoFs
  CU(zero_async(h, h->w2, sizeof(double) * N, h->stream));
  k_learned_guess<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->dims, stride, c[0], c[1], c[2], h->w2,
                                                     h->w2, h->nn_buf + 3 * nc, a, h->w1);
  ++h->launches;
  double alpha = 1.0;
  if (line_search) {
    // alpha = argmin |r(LE) - alpha J d| with the operator linearised at the extrapolation
    TRY(ensure_dt(h));
    const double *keepT = h->T_lin, *keepTo = h->T_old;
    h->T_lin = guess;
    h->T_old = T;
    h->lin_f_dirty = true;
    h->tf_dirty = true;
    h->tk_dirty = true;
    CU(zero_async(h, h->w2, sizeof(double) * N, h->stream));
    int rr = create_rhs(h, h->w2, T, heat_source);               // r = -R(LE)
    if (rr == MPDG_OK) {
      CU(zero_async(h, h->w3, sizeof(double) * N, h->stream));
      rr = op_apply_d(h, h->w3, h->w1, FIN_NONE, nullptr, nullptr);  // J d
    }
    h->T_lin = keepT;
    h->T_old = keepTo;
    h->lin_f_dirty = true;
    h->tf_dirty = true;
    h->tk_dirty = true;
    TRY(rr);
    double jj = 0.0, rj_plus = 0.0;
    TRY(norms(h, h->w3, nullptr, &jj, nullptr));
    TRY(norms(h, h->w2, h->w3, nullptr, &rj_plus));  // |r + Jd|^2
    double r2 = 0.0;
    TRY(norms(h, h->w2, nullptr, &r2, nullptr));
    const double rj = 0.5 * (rj_plus - r2 - jj);
    alpha = jj > 0.0 ? rj / jj : 0.0;
  }
  k_lincomb<<<vgrid(h, N), VT, 0, h->stream>>>(N, guess, 1.0, guess, alpha, h->w1);
  ++h->launches;
  CU(cudaGetLastError());
  if (alpha_out) *alpha_out = alpha;
  return distribute(h, guess);
}

extern "C" int mpdg_heat_learned_direction(mpdg_heat *h, mpdg_unet *u, int stride,
                                           const double *T, const double *T_old,
                                           const double *heat_source, double dt, double T_scale,
                                           double *direction)
{
  if (!h || !u || !T || !T_old || !direction)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (!(dt > 0.0) || !(T_scale > 0.0)) return fail(MPDG_ERR_INVALID_ARGUMENT, "dt and T_scale must be > 0");
  int c[3];
  TRY(learned_dims(h, stride, c));
  int ud[3];
  TRY(mpdg_unet_dims(u, ud));
  if (ud[0] != c[0] || ud[1] != c[1] || ud[2] != c[2])
    return fail(MPDG_ERR_INVALID_ARGUMENT, "network grid does not match the sampled mesh grid");
  CU(cudaSetDevice(h->device));
  const int64_t N = h->n_dofs;
  const int64_t nc = (int64_t)c[0] * c[1] * c[2];
  TRY(dalloc(h, reinterpret_cast<void **>(&h->nn_buf), sizeof(float) * 4 * nc));
  if (h->nn_buf_n == 0) h->nn_buf_n = nc;
  if (h->nn_buf_n != nc) return fail(MPDG_ERR_INVALID_ARGUMENT, "network grid changed");
  // per-sample scale: RMS of the time increment, kept on the device (no host round trip: the
  // feature and direction kernels take the square root themselves; a zero increment gives
  // zero features and a zero direction)
  k_diff_sq<<<vgrid(h, N), VT, 0, h->stream>>>(N, T, T_old, h->partials, h->counter, h->scal);
  ++h->launches;
  CU(cudaGetLastError());
  k_learned_input<<<vgrid(h, nc), VT, 0, h->stream>>>(h->dims, stride, c[0], c[1], c[2], T, T_old,
                                                     heat_source, dt, 1.0, 1.0, T_scale, h->scal,
                                                     1.0 / (double)N, h->nn_buf);
  ++h->launches;
  CU(cudaGetLastError());
  mpdg_unet_set_stream(u, h->stream);
  const int rc = mpdg_unet_forward(u, h->nn_buf, h->nn_buf + 3 * nc);
  if (rc != MPDG_OK) return fail(rc, "network forward failed");
  k_learned_direction<<<vgrid(h, N), VT, 0, h->stream>>>(N, h->dims, stride, c[0], c[1], c[2],
                                                         h->nn_buf + 3 * nc, 0.0, h->scal,
                                                         1.0 / (double)N, direction);
  ++h->launches;
  CU(cudaGetLastError());
  return MPDG_OK;
}
