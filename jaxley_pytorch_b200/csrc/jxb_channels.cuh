// Channel models of the step kernels: gating rates, exponential-Euler updates and
// ohmic currents, written once for a scalar type S (float, double, or a Dual of
// them for the adjoint's derivative with respect to the voltage).
//
// Each rate function restates the reference class at the cited line
// (jaxley-pytorch). Type ids match jaxley_pytorch_b200/channels.py.
#pragma once
#include "jxb_math.cuh"

namespace jxb {

enum ChannelType {
  CH_HH = 0, CH_LEAK = 1, CH_NATAT = 2, CH_NATS2T = 3, CH_NAPET2 = 4, CH_KPST = 5,
  CH_KTST = 6, CH_SKE2 = 7, CH_SKV3_1 = 8, CH_M = 9, CH_CAHVA = 10, CH_CALVA = 11,
  CH_CAPUMP = 12, CH_CANERNST = 13, CH_H = 14,
  // channels/pospischil.py: Na, K, Km, CaL, CaT
  CH_PNA = 15, CH_PK = 16, CH_PKM = 17, CH_PCAL = 18, CH_PCAT = 19
};

// One channel of a node class: its type and the node-relative slots of its states
// (role order of the reference's `channel_states`), of its current state and of its
// parameters (role order of `channel_params`, then `channel_constants`).
struct ChanEntry {
  short type, ns, np, cur;
  short s[6];
  short p[8];
};

enum GateId {
  G_HH_M, G_HH_H, G_HH_N, G_NATAT_M, G_NATAT_H, G_NATS2T_M, G_NATS2T_H, G_NAP_M,
  G_NAP_H, G_KPST_M, G_KPST_H, G_KTST_M, G_KTST_H, G_SKV31_M, G_M_M, G_CAHVA_M,
  G_CAHVA_H, G_CALVA_M, G_CALVA_H, G_H_M,
  G_PNA_M, G_PNA_H, G_PK_N, G_PKM_P, G_PCAL_Q, G_PCAL_R, G_PCAT_U
};

// Gates in alpha/beta form (`solve_gate_exponential`, solver_gate.py:45-53) versus
// x_inf/tau form (`solve_inf_gate_exponential`, solver_gate.py:67-87).
__device__ __forceinline__ bool gate_is_alpha_beta(int g) {
  return g == G_HH_M || g == G_HH_H || g == G_HH_N || g == G_CAHVA_M || g == G_CAHVA_H ||
         g == G_PNA_M || g == G_PNA_H || g == G_PK_N || g == G_PCAL_Q || g == G_PCAL_R;
}

template <typename S> struct Pair { S a, b; };

// Rates of every gate: (alpha, beta) for the alpha/beta gates, (x_inf, 1/tau) for the
// x_inf/tau gates. Each is the reference's expression with divisions by constants
// turned into products and u / (1 - exp(-u/k)) written as x_over_expm1(-u, k)
// (equal values; finite at u = 0 where the reference divides 0 by 0).
template <typename S>
__device__ __forceinline__ Pair<S> gate_rates(int g, S v) {
  typedef typename Base<S>::type B;
  const B qt = B(2.952882641412121);  // 2.3 ** ((34 - 21) / 10), l5pc.py
  Pair<S> r;
  switch (g) {
    case G_HH_M:  // channels/hh.py:88-92
      r.a = B(0.1) * x_over_expm1(-(v + B(40)), B(10));
      r.b = B(4.0) * save_exp(-(v + B(65)) * B(1.0 / 18.0));
      break;
    case G_HH_H:  // channels/hh.py:94-98
      r.a = B(0.07) * save_exp(-(v + B(65)) * B(1.0 / 20.0));
      r.b = rcp(save_exp(-(v + B(35)) * B(0.1)) + B(1));
      break;
    case G_HH_N:  // channels/hh.py:100-104
      r.a = B(0.01) * x_over_expm1(-(v + B(55)), B(10));
      r.b = B(0.125) * save_exp(-(v + B(65)) * B(1.0 / 80.0));
      break;
    case G_NATAT_M:
    case G_NATS2T_M: {  // l5pc.py:95-103, 177-185
      const B off = g == G_NATAT_M ? B(38) : B(32);
      S alpha = B(0.182) * x_over_expm1(-(v + off + B(1e-6)), B(6));
      S beta = B(0.124) * x_over_expm1(-(-v - off + B(1e-6)), B(6));
      S sum = alpha + beta;
      r.a = fdiv(alpha, sum);
      r.b = sum * qt;
      break;
    }
    case G_NATAT_H:
    case G_NATS2T_H: {  // l5pc.py:105-113, 187-195
      const B off = g == G_NATAT_H ? B(66) : B(60);
      S alpha = B(0.015) * x_over_expm1(v + off + B(1e-6), B(6));
      S beta = B(0.015) * x_over_expm1(-v - off + B(1e-6), B(6));
      S sum = alpha + beta;
      r.a = fdiv(alpha, sum);
      r.b = sum * qt;
      break;
    }
    case G_NAP_M: {  // l5pc.py:268-276
      S alpha = B(0.182) * x_over_expm1(-(v + B(38) + B(1e-6)), B(6));
      S beta = B(0.124) * x_over_expm1(-(-v - B(38) + B(1e-6)), B(6));
      r.b = (alpha + beta) * (qt * B(1.0 / 6.0));
      r.a = rcp(B(1) + save_exp((v + B(52.6)) * B(-1.0 / 4.6)));
      break;
    }
    case G_NAP_H: {  // l5pc.py:278-289
      S alpha = B(2.88e-6) * x_over_expm1(v + B(17) + B(1e-6), B(4.63));
      S w = -(v + B(64.4)) + B(1e-6);
      S beta = fdiv(B(-6.94e-6) * (v + B(64.4) + B(1e-6)), exm1(clamp20(w * B(1.0 / 2.63))));
      r.b = (alpha + beta) * qt;
      r.a = rcp(B(1) + save_exp((v + B(48.8)) * B(0.1)));
      break;
    }
    case G_KPST_M: {  // l5pc.py:355-369
      S va = v + B(10);
      r.a = rcp(B(1) + save_exp(-(va + B(1)) * B(1.0 / 12.0)));
      if (val(va) < B(-50.0))
        r.b = fdiv(S(qt), B(1.25) + B(175.03) * save_exp(va * B(0.026)));
      else
        r.b = fdiv(S(qt), B(1.25) + B(13) * save_exp(-va * B(0.026)));
      break;
    }
    case G_KPST_H: {  // l5pc.py:371-381
      S va = v + B(10);
      r.a = rcp(B(1) + save_exp((va + B(54)) * B(1.0 / 11.0)));
      S q = (va + B(75)) * B(1.0 / 48.0);
      r.b = fdiv(S(qt), B(360) + (B(1010) + B(24) * (va + B(55))) * save_exp(-(q * q)));
      break;
    }
    case G_KTST_M: {  // l5pc.py:444-451
      S va = v + B(10);
      r.a = rcp(B(1) + save_exp(-(va + B(0)) * B(1.0 / 19.0)));
      S q = (va + B(71)) * B(1.0 / 59.0);
      r.b = fdiv(S(qt), B(0.34) + B(0.92) * save_exp(-(q * q)));
      break;
    }
    case G_KTST_H: {  // l5pc.py:453-460
      S va = v + B(10);
      r.a = rcp(B(1) + save_exp((va + B(66)) * B(0.1)));
      S q = (va + B(73)) * B(1.0 / 23.0);
      r.b = fdiv(S(qt), B(8) + B(49) * save_exp(-(q * q)));
      break;
    }
    case G_SKV31_M:  // l5pc.py:585-590
      r.a = rcp(B(1) + save_exp((v - B(18.7)) * B(-1.0 / 9.7)));
      r.b = (B(1) + save_exp((v + B(46.56)) * B(-1.0 / 44.14))) * B(1.0 / (0.2 * 20.0));
      break;
    case G_M_M: {  // l5pc.py:653-661
      S ma = B(3.3e-3) * save_exp(B(2.5) * B(0.04) * (v + B(35)));
      S mb = B(3.3e-3) * save_exp(B(-2.5) * B(0.04) * (v + B(35)));
      S sum = ma + mb;
      r.a = fdiv(ma, sum);
      r.b = sum * qt;
      break;
    }
    case G_CAHVA_M:  // l5pc.py:723-727
      r.a = B(0.055) * x_over_expm1(B(-27) - v + B(1e-6), B(3.8));
      r.b = B(0.94) * save_exp((B(-75.0) - v + B(1e-6)) * B(1.0 / 17.0));
      break;
    case G_CAHVA_H:  // l5pc.py:729-734
      r.a = B(0.000457) * save_exp((B(-13.0) - v) * B(1.0 / 50.0));
      r.b = fdiv(S(B(0.0065)), save_exp((-v - B(15.0)) * B(1.0 / 28.0)) + B(1.0));
      break;
    case G_CALVA_M: {  // l5pc.py:795-802
      S vs = v + B(10);
      r.a = rcp(B(1) + save_exp((vs + B(30)) * B(-1.0 / 6.0)));
      r.b = fdiv(S(qt), B(5.0) + B(20.0) * rcp(B(1) + save_exp((vs + B(25)) * B(0.2))));
      break;
    }
    case G_CALVA_H: {  // l5pc.py:804-811
      S vs = v + B(10);
      r.a = rcp(B(1) + save_exp((vs + B(80)) * B(1.0 / 6.4)));
      r.b = fdiv(S(qt), B(20.0) + B(50.0) * rcp(B(1) + save_exp((vs + B(40)) * B(1.0 / 7.0))));
      break;
    }
    // channels/pospischil.py. The Na and K gates take v - vt and the CaT gate v + vx
    // (their parameters), passed as `v` by the caller; efun(x) = x_over_expm1(x, 1).
    case G_PNA_M:  // pospischil.py:124-131
      r.a = B(0.32) * x_over_expm1(B(-0.25) * (v - B(13)), B(1)) * B(4);
      r.b = B(0.28) * x_over_expm1(B(0.2) * (v - B(40)), B(1)) * B(5);
      break;
    case G_PNA_H:  // pospischil.py:133-140
      r.a = B(0.128) * save_exp(-(v - B(17)) * B(1.0 / 18.0));
      r.b = fdiv(S(B(4)), save_exp(-(v - B(40)) * B(0.2)) + B(1));
      break;
    case G_PK_N:  // pospischil.py:186-193
      r.a = B(0.032) * x_over_expm1(B(-0.2) * (v - B(15)), B(1)) * B(5);
      r.b = B(0.5) * save_exp(-(v - B(10)) * B(1.0 / 40.0));
      break;
    case G_PKM_P: {  // pospischil.py:242-249: (p_inf, 1 / tau * taumax); the caller scales
      S vp = v + B(35);
      r.a = rcp(B(1) + save_exp(B(-0.1) * vp));
      r.b = B(3.3) * save_exp(B(0.05) * vp) + save_exp(B(-0.05) * vp);
      break;
    }
    case G_PCAL_Q:  // pospischil.py:301-308
      r.a = B(0.055) * x_over_expm1((-v - B(27)) * B(1.0 / 3.8), B(1)) * B(3.8);
      r.b = B(0.94) * save_exp((-v - B(75)) * B(1.0 / 17.0));
      break;
    case G_PCAL_R:  // pospischil.py:310-317
      r.a = B(0.000457) * save_exp((-v - B(13)) * B(1.0 / 50.0));
      r.b = fdiv(S(B(0.0065)), save_exp((-v - B(15)) * B(1.0 / 28.0)) + B(1));
      break;
    case G_PCAT_U: {  // pospischil.py:366-375 (u_inf, 1 / tau)
      r.a = rcp(B(1) + save_exp((v + B(81)) * B(0.25)));
      S den = B(3.7) * (B(1) + save_exp((v + B(84)) * B(1.0 / 3.2)));
      r.b = fdiv(den, B(30.8) + (B(211.4) + save_exp((v + B(113.2)) * B(0.2))));
      break;
    }
    default: {  // G_H_M, l5pc.py:973-984
      S ma = B(0.001 * 6.43) * x_over_expm1(v + B(154.9) + B(1e-6), B(11.9));
      S mb = B(0.001 * 193) * save_exp(v * B(1.0 / 33.1));
      S sum = ma + mb;
      r.a = fdiv(ma, sum);
      r.b = sum;
      break;
    }
  }
  return r;
}

// exp(min(arg, 20)) - 1, the decay factor of exponential Euler minus one.
template <typename S> __device__ __forceinline__ S save_expm1(S x) { return exm1(clamp20(x)); }

// One exponential-Euler gate step. Returns x'; `e` receives d x'/d x.
// x * e + x_inf * (1 - e) (solver_gate.py:56-64) is evaluated as
// x + (x - x_inf) * (e - 1) with e - 1 from expm1: the same value, without the
// cancellation of 1 - e for slow gates in float32. `rate_scale` multiplies the
// 1 / tau of an x_inf/tau gate (Km's 1 / taumax).
template <typename S, typename B>
__device__ __forceinline__ S gate_step(int g, S v, B x, B dt, B* e_out, S rate_scale = S(B(1))) {
  Pair<S> r = gate_rates<S>(g, v);
  if (!gate_is_alpha_beta(g)) r.b = r.b * rate_scale;
  S xinf, em1;
  if (gate_is_alpha_beta(g)) {  // solver_gate.py:45-53: tau = 1/(a+b), x_inf = a*tau
    S sum = r.a + r.b;
    xinf = fdiv(r.a, sum);
    em1 = save_expm1(-dt * sum);
  } else {  // solver_gate.py:67-87: slope = -1/tau
    em1 = save_expm1(-r.b * dt);
    xinf = r.a;
  }
  if (e_out) *e_out = B(1) + val(em1);
  return x + (x - xinf) * em1;
}

// Steady state of a gate (`init_state` of the channel classes).
template <typename B>
__device__ __forceinline__ B gate_steady(int g, B v) {
  Pair<B> r = gate_rates<B>(g, v);
  if (gate_is_alpha_beta(g)) return fdiv(r.a, r.a + r.b);
  return r.a;
}

// `init_state` of the Pospischil Km and CaT gates (pospischil.py:232-237, 360-364),
// which pass their (x_inf, tau) pair to the alpha / (alpha + beta) of the alpha/beta
// gates: x_inf / (x_inf + tau). `tau_scale` is Km's taumax (1 for CaT).
template <typename B>
__device__ __forceinline__ B gate_init_inf_tau(int g, B v, B tau_scale) {
  Pair<B> r = gate_rates<B>(g, v);
  const B tau = tau_scale / r.b;
  return r.a / (r.a + tau);
}

// The CaT activation s_inf(v + vx) of its current (pospischil.py:350-357).
template <typename S>
__device__ __forceinline__ S pcat_sinf(S w) {
  typedef typename Base<S>::type B;
  return rcp(B(1) + save_exp(-(w + B(57)) * B(1.0 / 6.2)));
}

// SKE2 z gate, a function of the calcium concentration (l5pc.py:519-530).
template <typename S>
__device__ __forceinline__ S ske2_zinf(S cai) {
  typedef typename Base<S>::type B;
  if (val(cai) < B(1e-7)) cai = cai + B(1e-7);
  return rcp(B(1) + pw(fdiv(S(B(0.00043)), cai), B(4.8)));
}

// Gate ids and exponents of the gated ohmic channels.
struct GateLayout { int g0, g1, e0; };
__device__ __forceinline__ GateLayout gate_layout(int type) {
  switch (type) {
    case CH_NATAT: return {G_NATAT_M, G_NATAT_H, 3};
    case CH_NATS2T: return {G_NATS2T_M, G_NATS2T_H, 3};
    case CH_NAPET2: return {G_NAP_M, G_NAP_H, 3};
    case CH_KPST: return {G_KPST_M, G_KPST_H, 2};
    case CH_KTST: return {G_KTST_M, G_KTST_H, 4};
    case CH_CAHVA: return {G_CAHVA_M, G_CAHVA_H, 2};
    case CH_CALVA: return {G_CALVA_M, G_CALVA_H, 2};
    case CH_SKV3_1: return {G_SKV31_M, -1, 1};
    case CH_M: return {G_M_M, -1, 1};
    case CH_H: return {G_H_M, -1, 1};
    case CH_PNA: return {G_PNA_M, G_PNA_H, 3};
    case CH_PK: return {G_PK_N, -1, 4};
    case CH_PKM: return {G_PKM_P, -1, 1};
    case CH_PCAL: return {G_PCAL_Q, G_PCAL_R, 2};
    case CH_PCAT: return {G_PCAT_U, -1, 1};
    default: return {-1, -1, 0};
  }
}

template <typename B> __device__ __forceinline__ B ipow(B x, int n) {
  B r = x;
  for (int i = 1; i < n; ++i) r *= x;
  return r;
}

}  // namespace jxb
