// Host launchers of the cell kernels for one polynomial degree. Each
// cells_pN.cu translation unit includes this header and instantiates
// MPDG_DEFINE_DEGREE(n) so the degrees compile in parallel; the handle code
// reaches them through DegreeTable.
#pragma once

#include "cell_kernels.cuh"
#include "cell_kernels_v2.cuh"
#include "cell_kernels_f2.cuh"
#include "cell_kernels_tc.cuh"
#include "degree_table.hpp"

#include <stdlib.h>
#include <algorithm>
#include <type_traits>

namespace mpdg {

template <typename K>
static int persistent_grid(K kernel, int threads, size_t smem, int64_t n_batches, int sm_count,
                           int *cache)
{
  if (*cache <= 0) {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    *cache = per_sm > 0 ? per_sm : 1;
  }
  int64_t g = (int64_t)(*cache) * sm_count;
  if (g > n_batches) g = n_batches;
  if (g < 1) g = 1;
  return (int)g;
}

// FP32 operator on the scalar register-resident kernel (default) or the packed-pair
// kernel (MPDG_FP32_PACKED=1); both compute the same operator. The packed kernel
// issues 31 % fewer instructions at p = 3, but a packed FMA occupies the FMA pipe
// for two cycles and its 210-255 registers per lane halve the resident warps, so
// it measured 1.3-1.5x slower (p = 2, 3; constant k, k(T) tangent, Picard).
static inline bool fp32_packed()
{
  static const int on = [] {
    const char *e = getenv("MPDG_FP32_PACKED");
    return (e && e[0] == '1') ? 1 : 0;
  }();
  return on != 0;
}

// Register-resident operator on deformed meshes, p <= 2: a thread's 7 x n^2 geometry factors
// preloaded when the cell group starts or loaded in the quadrature-point loop. Mode 1 (the
// default) preloads where it measured faster: the k(T) tangents (FP64 1.4-1.5x, FP32
// 1.4-2.4x at p = 1, 2) and every FP64 law at p = 1 (1.12x); the constant-coefficient and
// Picard FP32 operators keep the loop loads (the preload measured up to 15 % slower there).
// MPDG_GEO_PRELOAD_V2=0 never preloads, =1 everywhere eligible.
static inline int geo_preload_v2()
{
  static const int mode = [] {
    const char *e = getenv("MPDG_GEO_PRELOAD_V2");
    return !e ? 1 : (e[0] == '0' ? 0 : (e[0] == '1' ? 2 : 1));
  }();
  return mode;
}
template <int n, typename T, int LAW> constexpr bool geo_preload_v2_default()
{
  return (sizeof(T) == 8 && n == 2) || LAW == 1 || LAW == 2 || LAW == 7;
}

// Line-per-thread operator on deformed meshes: the batch's per-point geometry
// preloaded into registers (default) or loaded in the quadrature-point loop
// (MPDG_GEO_PRELOAD=0); both compute the same operator.
static inline bool geo_preload()
{
  static const int on = [] {
    const char *e = getenv("MPDG_GEO_PRELOAD");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return on != 0;
}

template <int n>
struct DegreeOps {
  static constexpr int CPB = cells_per_block(n);
  static constexpr int THREADS = block_threads(n);

  static void upload(const double *tab, const float *tabf, const double *w, const float *wf)
  {
    cudaMemcpyToSymbol(c_tab_d, tab, sizeof(double) * kTabSize);
    cudaMemcpyToSymbol(c_tab_f, tabf, sizeof(float) * kTabSize);
    float2 tabf2[kTabSize];
    for (int i = 0; i < kTabSize; ++i) tabf2[i] = make_float2(tabf[i], tabf[i]);
    cudaMemcpyToSymbol(c_tab_f2, tabf2, sizeof(float2) * kTabSize);
    cudaMemcpyToSymbol(c_w_d, w, sizeof(double) * kWSize);
    cudaMemcpyToSymbol(c_w_f, wf, sizeof(float) * kWSize);
  }

  // register-resident kernel where a cell's planes fit the register file (FP64 at
  // p = 4 spills 64-750 bytes there and measured no faster than the line-per-thread
  // kernel on the deformed mesh, so it stays on the latter); the three-phase / transport
  // law with temperature dependence (LAW 5) runs the line-per-thread kernel
  template <typename T, int LAW = 0>
  static constexpr bool use_v2()
  {
    return LAW != 5 && (sizeof(T) == 8 ? n <= 4 : n <= 5);
  }

  template <typename T, int GEO, int LAW>
  static cudaError_t vmult_t(const CellArgs<T> &a, cudaStream_t s, int sm)
  {
    if constexpr (std::is_same<T, float>::value && n <= 4 && (LAW == 0 || LAW == 1 || LAW == 3)) {
      if (fp32_packed()) {
        static int cachep = 0;
        auto kp = k_vmult2p<n, GEO, LAW>;
        const size_t smemp = v2_smem<n, F2, LAW>();
        const int64_t ng = ((a.n_cells + 1) / 2 + v2_cells_per_warp<n>() - 1) / v2_cells_per_warp<n>();
        const int gp = persistent_grid(kp, 32 * kV2Warps, smemp, (ng + kV2Warps - 1) / kV2Warps,
                                       sm, &cachep);
        kp<<<gp, 32 * kV2Warps, smemp, s>>>(a);
        return cudaGetLastError();
      }
    }
    if constexpr (use_v2<T, LAW>()) {
      if constexpr (GEO == 1 && n <= 3) {
        const int mode = geo_preload_v2();
        if (mode == 2 || (mode == 1 && geo_preload_v2_default<n, T, LAW>())) {
          static int cachep = 0;
          auto kp = k_vmult2<n, T, GEO, LAW, true>;
          const size_t smemp = v2_smem<n, T, LAW>();
          const int64_t ng = (a.n_cells + v2_cells_per_warp<n>() - 1) / v2_cells_per_warp<n>();
          const int gp = persistent_grid(kp, 32 * kV2Warps, smemp, (ng + kV2Warps - 1) / kV2Warps,
                                         sm, &cachep);
          kp<<<gp, 32 * kV2Warps, smemp, s>>>(a);
          return cudaGetLastError();
        }
      }
      static int cache2 = 0;
      auto k2 = k_vmult2<n, T, GEO, LAW>;
      const size_t smem2 = v2_smem<n, T, LAW>();
      const int64_t ng = (a.n_cells + v2_cells_per_warp<n>() - 1) / v2_cells_per_warp<n>();
      const int g2 = persistent_grid(k2, 32 * kV2Warps, smem2, (ng + kV2Warps - 1) / kV2Warps, sm,
                                     &cache2);
      k2<<<g2, 32 * kV2Warps, smem2, s>>>(a);
      return cudaGetLastError();
    } else {
      const size_t smem = smem_vmult<n, T, LAW>();
      const int64_t nb = (a.n_cells + CPB - 1) / CPB;
      if constexpr (GEO == 1) {
        if (geo_preload()) {
          static int cachep = 0;
          auto kp = k_vmult<n, T, GEO, LAW, true>;
          const int g = persistent_grid(kp, THREADS, smem, nb, sm, &cachep);
          kp<<<g, THREADS, smem, s>>>(a);
          return cudaGetLastError();
        }
      }
      static int cache = 0;
      auto k = k_vmult<n, T, GEO, LAW>;
      const int g = persistent_grid(k, THREADS, smem, nb, sm, &cache);
      k<<<g, THREADS, smem, s>>>(a);
      return cudaGetLastError();
    }
  }
  template <typename T>
  static cudaError_t vmult(const CellArgs<T> &a, int geo, int law, cudaStream_t s, int sm)
  {
    if (law == 3) {
      if constexpr (use_v2<T>()) {
        return geo == 0 ? vmult_t<T, 0, 3>(a, s, sm) : vmult_t<T, 1, 3>(a, s, sm);
      } else {
        return cudaErrorNotSupported;
      }
    }
    if (law == 8) {  // the Picard operator from the gathered T_lin (linear-k law)
      if constexpr (use_v2<T>()) {
        return geo == 0 ? vmult_t<T, 0, 8>(a, s, sm) : vmult_t<T, 1, 8>(a, s, sm);
      } else {
        return cudaErrorNotSupported;
      }
    }
    if (law == 4) return geo == 0 ? vmult_t<T, 0, 4>(a, s, sm) : vmult_t<T, 1, 4>(a, s, sm);
    if (law == 5) return geo == 0 ? vmult_t<T, 0, 5>(a, s, sm) : vmult_t<T, 1, 5>(a, s, sm);
    if (law == 7) return geo == 0 ? vmult_t<T, 0, 7>(a, s, sm) : vmult_t<T, 1, 7>(a, s, sm);
    if (law == 6) {  // register-resident kernel only
      if constexpr (use_v2<T>()) {
        return geo == 0 ? vmult_t<T, 0, 6>(a, s, sm) : vmult_t<T, 1, 6>(a, s, sm);
      } else {
        return cudaErrorNotSupported;
      }
    }
    if (geo == 0) {
      if (law == 0) return vmult_t<T, 0, 0>(a, s, sm);
      if (law == 1) return vmult_t<T, 0, 1>(a, s, sm);
      return vmult_t<T, 0, 2>(a, s, sm);
    }
    if (law == 0) return vmult_t<T, 1, 0>(a, s, sm);
    if (law == 1) return vmult_t<T, 1, 1>(a, s, sm);
    return vmult_t<T, 1, 2>(a, s, sm);
  }
  static cudaError_t vmult_d(const CellArgs<double> &a, int geo, int law, cudaStream_t s, int sm)
  {
    return vmult<double>(a, geo, law, s, sm);
  }
  static cudaError_t vmult_f(const CellArgs<float> &a, int geo, int law, cudaStream_t s, int sm)
  {
    return vmult<float>(a, geo, law, s, sm);
  }

  template <int GEO, int LAW>
  static cudaError_t rhs_t(const CellArgs<double> &a, cudaStream_t s, int sm)
  {
    if constexpr (use_v2<double>() && (LAW == 0 || LAW == 1)) {
      static int cache2 = 0;
      auto k2 = k_rhs2<n, GEO, LAW>;
      const size_t smem2 =
        sizeof(double) * kV2Warps * 2 * (v2_cells_per_warp<n>() + 1) * v2_cell_stride<n>();
      const int64_t ng = (a.n_cells + v2_cells_per_warp<n>() - 1) / v2_cells_per_warp<n>();
      const int g2 = persistent_grid(k2, 32 * kV2Warps, smem2, (ng + kV2Warps - 1) / kV2Warps, sm,
                                     &cache2);
      k2<<<g2, 32 * kV2Warps, smem2, s>>>(a);
      return cudaGetLastError();
    }
    static int cache = 0;
    auto k = k_rhs<n, GEO, LAW>;
    const size_t smem = smem_rhs<n>();
    const int g = persistent_grid(k, THREADS, smem, (a.n_cells + CPB - 1) / CPB, sm, &cache);
    k<<<g, THREADS, smem, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t rhs(const CellArgs<double> &a, int geo, int law, cudaStream_t s, int sm)
  {
    if (law == 4) return geo == 0 ? rhs_t<0, 4>(a, s, sm) : rhs_t<1, 4>(a, s, sm);
    if (law == 5) return geo == 0 ? rhs_t<0, 5>(a, s, sm) : rhs_t<1, 5>(a, s, sm);
    if (geo == 0) {
      if (law == 0) return rhs_t<0, 0>(a, s, sm);
      if (law == 1) return rhs_t<0, 1>(a, s, sm);
      return rhs_t<0, 2>(a, s, sm);
    }
    if (law == 0) return rhs_t<1, 0>(a, s, sm);
    if (law == 1) return rhs_t<1, 1>(a, s, sm);
    return rhs_t<1, 2>(a, s, sm);
  }

  template <int GEO, int LAW>
  static cudaError_t diag_t(const CellArgs<double> &a, cudaStream_t s, int sm)
  {
    static int cache = 0;
    auto k = k_diag<n, GEO, LAW>;
    const size_t smem = smem_diag<n>();
    const int g = persistent_grid(k, THREADS, smem, (a.n_cells + CPB - 1) / CPB, sm, &cache);
    k<<<g, THREADS, smem, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t diag(const CellArgs<double> &a, int geo, int law, cudaStream_t s, int sm)
  {
    if (law == 4) return geo == 0 ? diag_t<0, 4>(a, s, sm) : diag_t<1, 4>(a, s, sm);
    if (law == 5) return geo == 0 ? diag_t<0, 5>(a, s, sm) : diag_t<1, 5>(a, s, sm);
    if (geo == 0) {
      if (law == 0) return diag_t<0, 0>(a, s, sm);
      if (law == 1) return diag_t<0, 1>(a, s, sm);
      return diag_t<0, 2>(a, s, sm);
    }
    if (law == 0) return diag_t<1, 0>(a, s, sm);
    if (law == 1) return diag_t<1, 1>(a, s, sm);
    return diag_t<1, 2>(a, s, sm);
  }

  template <int GEO>
  static cudaError_t norm_t(const CellArgs<double> &a, cudaStream_t s, int sm)
  {
    static int cache = 0;
    auto k = k_norm<n, GEO>;
    const size_t smem = smem_norm<n>();
    const int g = persistent_grid(k, THREADS, smem, (a.n_cells + CPB - 1) / CPB, sm, &cache);
    k<<<g, THREADS, smem, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t norm(const CellArgs<double> &a, int geo, int, cudaStream_t s, int sm)
  {
    return geo == 0 ? norm_t<0>(a, s, sm) : norm_t<1>(a, s, sm);
  }

  template <int LAW>
  static cudaError_t kq_t(const CellArgs<double> &a, float *kq, cudaStream_t s, int sm)
  {
    static int cache = 0;
    auto k = k_conductivity_q<n, LAW>;
    const size_t smem = sizeof(double) * kV2Warps * (v2_cells_per_warp<n>() + 1) * v2_cell_stride<n>();
    const int64_t ng = (a.n_cells + v2_cells_per_warp<n>() - 1) / v2_cells_per_warp<n>();
    const int g = persistent_grid(k, 32 * kV2Warps, smem, (ng + kV2Warps - 1) / kV2Warps, sm, &cache);
    k<<<g, 32 * kV2Warps, smem, s>>>(a, kq);
    return cudaGetLastError();
  }
  template <int GEO>
  static cudaError_t diag_picard_t(const CellArgs<float> &a, cudaStream_t s, int sm)
  {
    static int cache = 0;
    auto k = k_diag_picard<n, GEO>;
    const size_t smem = sizeof(float) * kV2Warps * 2 * (v2_cells_per_warp<n>() + 1) * v2_cell_stride<n>();
    const int64_t ng = (a.n_cells + v2_cells_per_warp<n>() - 1) / v2_cells_per_warp<n>();
    const int g = persistent_grid(k, 32 * kV2Warps, smem, (ng + kV2Warps - 1) / kV2Warps, sm, &cache);
    k<<<g, 32 * kV2Warps, smem, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t diag_picard(const CellArgs<float> &a, int geo, cudaStream_t s, int sm)
  {
    return geo == 0 ? diag_picard_t<0>(a, s, sm) : diag_picard_t<1>(a, s, sm);
  }
  template <int GEO>
  static cudaError_t vmult_picard_rows_t(const CellArgs<float> &a, cudaStream_t s, int sm)
  {
    static int cache = 0;
    auto k = k_vmult2<n, float, GEO, 3, false, true>;
    const size_t smem = v2_smem<n, float, 3>();
    const int64_t ng = (a.n_cells + v2_cells_per_warp<n>() - 1) / v2_cells_per_warp<n>();
    const int g = persistent_grid(k, 32 * kV2Warps, smem, (ng + kV2Warps - 1) / kV2Warps, sm, &cache);
    k<<<g, 32 * kV2Warps, smem, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t vmult_picard_rows(const CellArgs<float> &a, int geo, cudaStream_t s, int sm)
  {
    if constexpr (n == 4) {
      return geo == 0 ? vmult_picard_rows_t<0>(a, s, sm) : vmult_picard_rows_t<1>(a, s, sm);
    } else {
      (void)a, (void)geo, (void)s, (void)sm;
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t vmult_picard_tc(const CellArgs<float> &a, const float *gmat, int *err,
                                     cudaStream_t s, int sm)
  {
    if constexpr (n == 4) {
      static bool attr = false;
      auto k = k_vmult_picard_tc<n>;
      if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)optc::kSmem);
        if (e != cudaSuccess) return e;
        attr = true;
      }
      const int64_t nb = (int64_t)((a.d.m[0] + optc::kBX - 1) / optc::kBX) *
                         ((a.d.m[1] + optc::kBY - 1) / optc::kBY) *
                         ((a.d.m[2] + optc::kBZ - 1) / optc::kBZ);
      // one CTA per SM (two brick pipelines, 512 tensor-memory columns, ~161 KB shared)
      const int64_t nc = (nb + optc::kGroups - 1) / optc::kGroups;
      const int g = (int)std::min<int64_t>(nc, (int64_t)sm);
      k<<<g, optc::kThreads, optc::kSmem, s>>>(a, reinterpret_cast<const float4 *>(gmat), err);
      return cudaGetLastError();
    } else {
      (void)a, (void)gmat, (void)err, (void)s, (void)sm;
      return cudaErrorNotSupported;
    }
  }
  template <int GEO>
  static cudaError_t coef_tangent_t(const CellArgs<double> &a, double *out, cudaStream_t s, int sm)
  {
    static int cache = 0;
    auto k = k_coef_tangent<n, GEO>;
    const size_t smem = smem_coef_tangent<n>();
    const int g = persistent_grid(k, THREADS, smem, (a.n_cells + CPB - 1) / CPB, sm, &cache);
    k<<<g, THREADS, smem, s>>>(a, out);
    return cudaGetLastError();
  }
  static cudaError_t coef_tangent(const CellArgs<double> &a, double *out, int geo, cudaStream_t s,
                                  int sm)
  {
    return geo == 0 ? coef_tangent_t<0>(a, out, s, sm) : coef_tangent_t<1>(a, out, s, sm);
  }
  template <int GEO>
  static cudaError_t coef_lineark_t(const CellArgs<double> &a, double *out, cudaStream_t s, int sm)
  {
    static int cache = 0;
    auto k = k_coef_lineark<n, GEO>;
    const size_t smem = smem_coef_lineark<n>();
    const int g = persistent_grid(k, THREADS, smem, (a.n_cells + CPB - 1) / CPB, sm, &cache);
    k<<<g, THREADS, smem, s>>>(a, out);
    return cudaGetLastError();
  }
  static cudaError_t coef_lineark(const CellArgs<double> &a, double *out, int geo, cudaStream_t s,
                                  int sm)
  {
    return geo == 0 ? coef_lineark_t<0>(a, out, s, sm) : coef_lineark_t<1>(a, out, s, sm);
  }
  static cudaError_t field_values(const CellArgs<double> &a, const double *H, const double *vel,
                                  int64_t n_dofs, double *cf, cudaStream_t s, int sm)
  {
    static int cache = 0;
    auto k = k_field_values<n>;
    const size_t smem = smem_norm<n>();
    const int g = persistent_grid(k, THREADS, smem, (a.n_cells + CPB - 1) / CPB, sm, &cache);
    k<<<g, THREADS, smem, s>>>(a, H, vel, n_dofs, cf);
    return cudaGetLastError();
  }
  static cudaError_t conductivity_q(const CellArgs<double> &a, float *kq, int law, cudaStream_t s,
                                    int sm)
  {
    if (law == 0) return kq_t<0>(a, kq, s, sm);
    if (law == 1) return kq_t<1>(a, kq, s, sm);
    return kq_t<2>(a, kq, s, sm);
  }

  static DegreeTable table()
  {
    DegreeTable t;
    t.n = n;
    t.upload = &upload;
    t.vmult_d = &vmult_d;
    t.vmult_f = &vmult_f;
    t.rhs = &rhs;
    t.diag = &diag;
    t.norm = &norm;
    t.coef_tangent = &coef_tangent;
    t.coef_lineark = &coef_lineark;
    t.field_values = &field_values;
    t.v2_d = use_v2<double>();
    t.v2_f = use_v2<float>();
    if constexpr (use_v2<float>()) {
      t.conductivity_q = &conductivity_q;
      t.diag_picard = &diag_picard;
    }
    if constexpr (n == 4) {
      t.vmult_picard_tc = &vmult_picard_tc;
      t.vmult_picard_rows = &vmult_picard_rows;
    }
    return t;
  }
};

}  // namespace mpdg

#define MPDG_DEFINE_DEGREE(N)                                            \
  namespace mpdg {                                                       \
  DegreeTable degree_table_##N() { return DegreeOps<N>::table(); }        \
  }
