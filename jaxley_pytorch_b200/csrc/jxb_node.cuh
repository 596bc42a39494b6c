// Per-node channel work of one step (forward), shared by the forward and the
// adjoint kernels.
#pragma once
#include "jxb_channels.cuh"

namespace jxb {

// Parameter accessor of one node and batch row: value = base * scale[col].
template <typename T>
struct Prm {
  const T* base;
  const int* col;
  const T* scale;
  __device__ __forceinline__ T operator()(int k) const { return base[k] * scale[col[k]]; }
};

// `update_states` of one channel entry, in place on the node's state block `x`
// (modules/base.py:3414-3443 calls them sequentially in insertion order).
template <typename T>
__device__ __forceinline__ void channel_update(const ChanEntry& e, T* x, const Prm<T>& P, T v,
                                               T dt) {
  switch (e.type) {
    case CH_HH:  // channels/hh.py:37-50
      x[e.s[0]] = gate_step<T, T>(G_HH_M, v, x[e.s[0]], dt, nullptr);
      x[e.s[1]] = gate_step<T, T>(G_HH_H, v, x[e.s[1]], dt, nullptr);
      x[e.s[2]] = gate_step<T, T>(G_HH_N, v, x[e.s[2]], dt, nullptr);
      break;
    case CH_LEAK:
      break;
    case CH_SKE2: {  // l5pc.py:488-500, tau_z = 1
      T zinf = ske2_zinf<T>(x[e.s[1]]);
      T ez = save_exp(T(-1.0) / T(1.0) * dt);
      x[e.s[0]] = x[e.s[0]] * ez + zinf * (T(1) - ez);
      break;
    }
    case CH_CAPUMP: {  // l5pc.py:842-861
      T ica = x[e.cur];
      T cai = x[e.s[0]];
      T gamma = P(0), decay = P(1), depth = P(2), minCai = P(3);
      T drive = T(-10000.0) * ica * gamma / (T(2) * T(96485) * depth);
      T cai_inf = minCai + decay * drive;
      T ee = save_exp(-dt / decay);
      x[e.s[0]] = cai * ee + cai_inf * (T(1) - ee);
      break;
    }
    case CH_CANERNST: {  // l5pc.py:891-902; constants F, T, R
      T F = P(0), Tk = P(1), R = P(2);
      T C = R * Tk / (T(2) * F) * T(1000);
      x[e.s[0]] = C * lg(x[e.s[2]] / x[e.s[1]]);
      break;
    }
    default: {  // gated ohmic channels (l5pc.py update_states)
      GateLayout gl = gate_layout(e.type);
      x[e.s[0]] = gate_step<T, T>(gl.g0, v, x[e.s[0]], dt, nullptr);
      if (gl.g1 >= 0) x[e.s[1]] = gate_step<T, T>(gl.g1, v, x[e.s[1]], dt, nullptr);
      break;
    }
  }
}

// `init_state` of one channel entry (steady state at the node voltage).
template <typename T>
__device__ __forceinline__ void channel_steady(const ChanEntry& e, T* x, T v) {
  switch (e.type) {
    case CH_HH:  // channels/hh.py:69-86
      x[e.s[0]] = gate_steady<T>(G_HH_M, v);
      x[e.s[1]] = gate_steady<T>(G_HH_H, v);
      x[e.s[2]] = gate_steady<T>(G_HH_N, v);
      break;
    case CH_SKE2:  // l5pc.py:513-517
      x[e.s[0]] = ske2_zinf<T>(T(5e-05));
      break;
    case CH_LEAK:
    case CH_CAPUMP:
    case CH_CANERNST:
      break;
    default: {
      GateLayout gl = gate_layout(e.type);
      x[e.s[0]] = gate_steady<T>(gl.g0, v);
      if (gl.g1 >= 0) x[e.s[1]] = gate_steady<T>(gl.g1, v);
      break;
    }
  }
}

// Conductance (without the maximal conductance) and reversal of the gated ohmic
// channels: I = g * G * (v - E).
template <typename T>
__device__ __forceinline__ T gated_G(const ChanEntry& e, const T* x, int e0, bool has_h) {
  T G = ipow(x[e.s[0]], e0);
  if (has_h) G *= x[e.s[1]];
  return G;
}

// `compute_current` of one entry, linearised: the reference's finite difference
// (modules/base.py:3505-3542) of a current that is linear in v is exactly
// slope = g*G and offset = -g*G*E; the unperturbed current is added to the
// current state slot.
template <typename T>
__device__ __forceinline__ void channel_current(const ChanEntry& e, T* x, const Prm<T>& P, T v,
                                                T& slope, T& gge) {
  T cur = T(0);
  switch (e.type) {
    case CH_HH: {  // channels/hh.py:52-67
      T m = x[e.s[0]], h = x[e.s[1]], n = x[e.s[2]];
      T gNa = P(0) * (m * m * m) * h;
      T gK = P(1) * (n * n * n * n);
      T gL = P(2);
      slope += gNa + gK + gL;
      gge += gNa * P(3) + gK * P(4) + gL * P(5);
      cur = gNa * (v - P(3)) + gK * (v - P(4)) + gL * (v - P(5));
      break;
    }
    case CH_LEAK: {  // channels/pospischil.py:64-68
      T g = P(0);
      slope += g;
      gge += g * P(1);
      cur = g * (v - P(1));
      break;
    }
    case CH_SKE2: {  // l5pc.py:502-511
      T g = P(0) * x[e.s[0]];
      slope += g;
      gge += g * P(1);
      cur = g * (v - P(1));
      break;
    }
    case CH_CAPUMP:
    case CH_CANERNST:
      return;
    default: {  // l5pc.py compute_current of the gated channels
      GateLayout gl = gate_layout(e.type);
      T g = P(0) * gated_G(e, x, gl.e0, gl.g1 >= 0);
      T E = (e.type == CH_CAHVA || e.type == CH_CALVA) ? x[e.s[2]] : P(1);
      slope += g;
      gge += g * E;
      cur = g * (v - E);
      break;
    }
  }
  x[e.cur] += cur;
}

}  // namespace jxb
