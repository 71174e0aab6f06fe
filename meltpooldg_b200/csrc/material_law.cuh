// Material laws of the heat operator at one point (Material::compute_parameters,
// include/meltpooldg/core/material.templates.hpp:104-137, 226-500), shared by the cell kernels
// and the host evaluator mpdg_material_eval: rho*cp, k and their temperature derivatives.
#pragma once

#include "cell_args.cuh"

#if defined(__CUDACC__)
#define MPDG_LAW_HD __host__ __device__ __forceinline__
#else
#define MPDG_LAW_HD inline
#endif

namespace mpdg {

// ramp from (x1, y1) to (x2, y2) with zero slope at both ends: quadratic over the first and the
// last `delta`, linear in between with the slope s = (y2 - y1) / (x2 - x1 - delta) at which the
// pieces meet with continuous slopes (qlq_zero_slope, source/heat/apparent_capacity.cpp:41-110);
// dy its derivative
template <typename T>
MPDG_LAW_HD T qlq_ramp(T x, T x1, T x2, T y1, T y2, T delta, T &dy)
{
  const T s = (y2 - y1) / (x2 - x1 - delta);
  if (x < x1 + delta) {
    dy = s / delta * (x - x1);
    return y1 + T(0.5) * s / delta * (x - x1) * (x - x1);
  }
  if (x > x2 - delta) {
    dy = -s / delta * (x - x2);
    return y2 - T(0.5) * s / delta * (x - x2) * (x - x2);
  }
  dy = s;
  return y1 + s * (x - x1 - T(0.5) * delta);
}

// apparent heat capacity of the latent heat of fusion L in the mushy zone, added to the
// liquid-solid specific heat capacity when L > 0 (Heat::ApparentCapacity,
// source/heat/apparent_capacity.cpp:157-300; material.templates.hpp:562-616): zero unless
// 0 < sf < 1; with dT = T_l - T_s each profile integrates to L over [T_s, T_l]:
//   acap 1 (constant)    L / dT
//   acap 0 (qlq)         qlq_ramp from (T_s, 0) up to (T_mid, 2 L / dT) and down to (T_l, 0),
//                        delta = dT / 6, at T = T_l - sf dT
//   acap 2 (poly4 bell)  (2 L / dT) f(xi), f(x) = 15/16 (x^2 - 1)^2, xi = 1 - 2 sf
// dA its temperature derivative
template <typename T>
MPDG_LAW_HD T apparent_capacity(const MatParams<T> &m, T sf, T &dA)
{
  dA = T(0);
  if (sf <= T(0) || sf >= T(1)) return T(0);
  const T L = m.latent, dT = m.T_liq - m.T_sol;
  if (m.acap == 1) return L / dT;
  if (m.acap == 2) {
    const T r = T(2) / dT, xi = T(1) - T(2) * sf, q = xi * xi - T(1);
    dA = L * r * r * T(3.75) * xi * q;
    return L * r * T(0.9375) * q * q;
  }
  const T Tq = m.T_liq - sf * dT, Tm = T(0.5) * (m.T_sol + m.T_liq);
  const T peak = T(2) * L / dT, delta = dT / T(6);
  return Tq <= Tm ? qlq_ramp(Tq, m.T_sol, Tm, T(0), peak, delta, dA)
                  : qlq_ramp(Tq, Tm, m.T_liq, peak, T(0), delta, dA);
}

// Material::compute_parameters for the three laws; LAW is a template constant.
template <int LAW, typename T>
MPDG_LAW_HD void mat_eval(const MatParams<T> &m, T temp, T &rhocp, T &k, T &drhocp, T &dk)
{
  if (LAW == 0) {
    rhocp = m.rho_l * m.cp_l;
    k = m.k_l;
    drhocp = T(0);
    dk = T(0);
  } else if (LAW == 1) {
    rhocp = m.rho_l * m.cp_l;
    k = m.k_l + m.k1 * temp;
    drhocp = T(0);
    dk = m.k1;
  } else {
    T sf;
    if (m.sharp)
      sf = temp < m.T_sol ? T(1) : T(0);
    else {
      sf = (m.T_liq - temp) * m.inv_mushy;
      sf = sf < T(0) ? T(0) : (sf > T(1) ? T(1) : sf);
    }
    const T hs = T(-2) * sf * sf * sf + T(3) * sf * sf;
    const T dhs = T(-6) * sf * sf + T(6) * sf;
    const bool edge = (sf == T(0) || sf == T(1));
    auto prop = [&](T l, T s) { return sf == T(0) ? l : (sf == T(1) ? s : l + (s - l) * hs); };
    auto dprop = [&](T l, T s) { return edge ? T(0) : T(-1) * m.inv_mushy * ((s - l) * dhs); };
    k = prop(m.k_l, m.k_s);
    dk = dprop(m.k_l, m.k_s);
    if (m.vs) {
      rhocp = prop(m.rho_l * m.cp_l, m.rho_s * m.cp_s);
      drhocp = dprop(m.rho_l * m.cp_l, m.rho_s * m.cp_s);
    } else {
      const T rho = prop(m.rho_l, m.rho_s), drho = dprop(m.rho_l, m.rho_s);
      T cp = prop(m.cp_l, m.cp_s), dcp = dprop(m.cp_l, m.cp_s);
      if (m.latent > T(0)) {
        T dA;
        cp += apparent_capacity(m, sf, dA);
        dcp += dA;
      }
      rhocp = rho * cp;
      drhocp = dcp * rho + drho * cp;
    }
  }
}

// Three-phase law (Material::compute_parameters, gas_liquid_solid,
// material.templates.hpp:376-500, 620-740): every property is (1 - w) gas + w ls(T) with
// ls the liquid-solid interpolation of mat_eval<2>, its T derivative w dls/dT; w = 1 gives
// the liquid-solid law exactly.
template <typename T>
MPDG_LAW_HD void mat_eval_w(const MatParams<T> &m, T temp, T w, T &rhocp, T &k, T &drhocp, T &dk)
{
  T sf;
  if (m.sharp)
    sf = temp < m.T_sol ? T(1) : T(0);
  else {
    sf = (m.T_liq - temp) * m.inv_mushy;
    sf = sf < T(0) ? T(0) : (sf > T(1) ? T(1) : sf);
  }
  const T hs = T(-2) * sf * sf * sf + T(3) * sf * sf;
  const T dhs = T(-6) * sf * sf + T(6) * sf;
  const bool edge = (sf == T(0) || sf == T(1));
  auto prop = [&](T l, T s) { return sf == T(0) ? l : (sf == T(1) ? s : l + (s - l) * hs); };
  auto dprop = [&](T l, T s) { return edge ? T(0) : T(-1) * m.inv_mushy * ((s - l) * dhs); };
  const T g = T(1) - w;
  k = g * m.k_g + w * prop(m.k_l, m.k_s);
  dk = w * dprop(m.k_l, m.k_s);
  if (m.vs) {
    rhocp = g * (m.rho_g * m.cp_g) + w * prop(m.rho_l * m.cp_l, m.rho_s * m.cp_s);
    drhocp = w * dprop(m.rho_l * m.cp_l, m.rho_s * m.cp_s);
  } else {
    T cpls = prop(m.cp_l, m.cp_s), dcpls = dprop(m.cp_l, m.cp_s);
    if (m.latent > T(0)) {
      T dA;
      cpls += apparent_capacity(m, sf, dA);
      dcpls += dA;
    }
    const T rho = g * m.rho_g + w * prop(m.rho_l, m.rho_s);
    const T cp = g * m.cp_g + w * cpls;
    drhocp = (w * dcpls) * rho + (w * dprop(m.rho_l, m.rho_s)) * cp;
    rhocp = rho * cp;
  }
}

}  // namespace mpdg
