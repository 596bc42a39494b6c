// Per-node channel work of one step (forward), shared by the forward and the
// adjoint kernels.
#pragma once
#include "jxb_channels.cuh"

namespace jxb {

// Parameter values of one channel entry of one node and batch row (staged in shared
// memory as base * scale[col] when the launch starts).
template <typename T>
struct Prm {
  const T* val;
  __device__ __forceinline__ T operator()(int k) const { return val[k]; }
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
      T em1 = save_expm1(T(-1.0) / T(1.0) * dt);
      T z = x[e.s[0]];
      x[e.s[0]] = z + (z - zinf) * em1;
      break;
    }
    case CH_CAPUMP: {  // l5pc.py:842-861
      T ica = x[e.cur];
      T cai = x[e.s[0]];
      T gamma = P(0), decay = P(1), depth = P(2), minCai = P(3);
      T drive = T(-10000.0) * ica * gamma / (T(2) * T(96485) * depth);
      T cai_inf = minCai + decay * drive;
      T em1 = save_expm1(-dt / decay);
      x[e.s[0]] = cai + (cai - cai_inf) * em1;
      break;
    }
    case CH_CANERNST: {  // l5pc.py:891-902; constants F, T, R
      T F = P(0), Tk = P(1), R = P(2);
      T C = R * Tk / (T(2) * F) * T(1000);
      x[e.s[0]] = C * lg(x[e.s[2]] / x[e.s[1]]);
      break;
    }
    case CH_PNA: {  // pospischil.py:91-104, gates of v - vt
      const T u = v - P(2);
      x[e.s[0]] = gate_step<T, T>(G_PNA_M, u, x[e.s[0]], dt, nullptr);
      x[e.s[1]] = gate_step<T, T>(G_PNA_H, u, x[e.s[1]], dt, nullptr);
      break;
    }
    case CH_PK:  // pospischil.py:158-169
      x[e.s[0]] = gate_step<T, T>(G_PK_N, v - P(2), x[e.s[0]], dt, nullptr);
      break;
    case CH_PKM:  // pospischil.py:212-225, tau = taumax / (...)
      x[e.s[0]] = gate_step<T, T>(G_PKM_P, v, x[e.s[0]], dt, nullptr, T(1) / P(1));
      break;
    case CH_PCAT:  // pospischil.py:334-347, gate of v + vx
      x[e.s[0]] = gate_step<T, T>(G_PCAT_U, v + P(1), x[e.s[0]], dt, nullptr);
      break;
    default: {  // gated ohmic channels (l5pc.py update_states; Pospischil CaL)
      GateLayout gl = gate_layout(e.type);
      x[e.s[0]] = gate_step<T, T>(gl.g0, v, x[e.s[0]], dt, nullptr);
      if (gl.g1 >= 0) x[e.s[1]] = gate_step<T, T>(gl.g1, v, x[e.s[1]], dt, nullptr);
      break;
    }
  }
}

// `init_state` of one channel entry (steady state at the node voltage).
template <typename T>
__device__ __forceinline__ void channel_steady(const ChanEntry& e, T* x, const Prm<T>& P, T v) {
  switch (e.type) {
    case CH_PNA:  // pospischil.py:117-125
      x[e.s[0]] = gate_steady<T>(G_PNA_M, v - P(2));
      x[e.s[1]] = gate_steady<T>(G_PNA_H, v - P(2));
      break;
    case CH_PK:  // pospischil.py:180-184
      x[e.s[0]] = gate_steady<T>(G_PK_N, v - P(2));
      break;
    case CH_PKM:  // pospischil.py:232-237
      x[e.s[0]] = gate_init_inf_tau<T>(G_PKM_P, v, P(1));
      break;
    case CH_PCAT:  // pospischil.py:360-364
      x[e.s[0]] = gate_init_inf_tau<T>(G_PCAT_U, v + P(1), T(1));
      break;
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
    case CH_PKM: {  // pospischil.py:227-230: E = eK, the third parameter
      T g = P(0) * x[e.s[0]];
      slope += g;
      gge += g * P(2);
      cur = g * (v - P(2));
      break;
    }
    case CH_PCAT: {  // pospischil.py:349-357: not linear in v, the reference's finite
      // difference of 1e-3 mV (modules/base.py:3522-3539) gives slope and offset
      const T g = P(0) * x[e.s[0]], vx = P(1), E = P(2);
      const T s0 = pcat_sinf<T>(v + vx), s1 = pcat_sinf<T>((v + T(1e-3)) + vx);
      const T i0 = g * (s0 * s0) * (v - E);
      const T i1 = g * (s1 * s1) * ((v + T(1e-3)) - E);
      const T vt = (i1 - i0) * T(1000.0);
      slope += vt;
      gge += vt * v - i0;
      cur = i0;
      break;
    }
    default: {  // l5pc.py compute_current of the gated channels; Pospischil Na, K, CaL
      GateLayout gl = gate_layout(e.type);
      T g = P(0) * gated_G(e, x, gl.e0, gl.g1 >= 0);
      T E = (e.type == CH_CAHVA || e.type == CH_CALVA) ? x[e.s[2]] : P(1);
      slope += g;
      gge += g * E;
      cur = g * (v - E);
      break;
    }
  }
  if (e.cur >= 0) x[e.cur] += cur;
}

}  // namespace jxb

namespace jxb {

// ---------------------------------------------------------------------------------
// Adjoint (vector-Jacobian products) of one node's channel step.
//
// `lam` is the node's adjoint block (same slot layout as the state); `lv` collects
// the adjoint of the node voltage before the step. Parameter adjoints go through
// `PGrad::add(k, value)` with `k` relative to the entry's first parameter.
// ---------------------------------------------------------------------------------

template <typename T>
struct PGradSink {
  // Accumulates d loss / d parameter value times the parameter base (the gradient of
  // the column scale) into the node's own slot of every trainable parameter
  // (gk >= 0), in the precision of the run; fixed parameters are skipped. No two
  // threads share a slot; the slots are folded into float64 columns once per launch.
  const T* base;
  const int* gk;
  T* acc;  // the node's gradient slots (shared memory)
  __device__ __forceinline__ void add(int k, T g) const {
    const int q = gk[k];
    if (q >= 0) acc[q] += g * base[k];
  }
};

// VJP of `channel_current` at the post-update state `x` and voltage `v`.
// The node's summed slope s and g*E term q enter the solve as
// d += dt * 1000 * s / cm and rhs += dt * 1000 * q / cm, so with
// lr = 1000 * dt * lambda_r / cm and the new voltage x1 their adjoints are
// -lr * x1 and lr; a conductance c with reversal E gets lr * (E - x1).
template <typename T>
__device__ __forceinline__ void channel_current_vjp(const ChanEntry& e, const T* x, T* lam,
                                                    const Prm<T>& P, const PGradSink<T>& G, T v,
                                                    T lr, T x1, T& lv) {
  const T lI = e.cur >= 0 ? lam[e.cur] : T(0);
  auto ohmic = [&](T c, T E, T& lc, T& lE) {
    lc = lr * (E - x1) + (v - E) * lI;
    lE = c * (lr - lI);
    lv += c * lI;
  };
  switch (e.type) {
    case CH_HH: {
      T m = x[e.s[0]], h = x[e.s[1]], n = x[e.s[2]];
      T G1 = (m * m * m) * h, G2 = (n * n * n * n);
      T gNa = P(0), gK = P(1), gL = P(2);
      T lc1, lE1, lc2, lE2, lc3, lE3;
      ohmic(gNa * G1, P(3), lc1, lE1);
      ohmic(gK * G2, P(4), lc2, lE2);
      ohmic(gL, P(5), lc3, lE3);
      lam[e.s[0]] += gNa * T(3) * m * m * h * lc1;
      lam[e.s[1]] += gNa * m * m * m * lc1;
      lam[e.s[2]] += gK * T(4) * n * n * n * lc2;
      G.add(0, G1 * lc1);
      G.add(1, G2 * lc2);
      G.add(2, lc3);
      G.add(3, lE1);
      G.add(4, lE2);
      G.add(5, lE3);
      break;
    }
    case CH_LEAK: {
      T lc, lE;
      ohmic(P(0), P(1), lc, lE);
      G.add(0, lc);
      G.add(1, lE);
      break;
    }
    case CH_SKE2: {
      T g = P(0), z = x[e.s[0]];
      T lc, lE;
      ohmic(g * z, P(1), lc, lE);
      lam[e.s[0]] += g * lc;
      G.add(0, z * lc);
      G.add(1, lE);
      break;
    }
    case CH_CAPUMP:
    case CH_CANERNST:
      break;
    case CH_PKM: {
      T g = P(0), p = x[e.s[0]];
      T lc, lE;
      ohmic(g * p, P(2), lc, lE);
      lam[e.s[0]] += g * lc;
      G.add(0, p * lc);
      G.add(2, lE);
      break;
    }
    case CH_PCAT: {
      // slope s = (i1 - i0) / d and offset q = s v - i0 of the finite difference,
      // with adjoints -lr x1 and lr; the current slot holds i0.
      const T d = T(1e-3);
      const T g = P(0), u = x[e.s[0]], vx = P(1), E = P(2);
      const Dual<T> a0 = pcat_sinf<Dual<T>>(Dual<T>(v + vx, T(1)));
      const Dual<T> a1 = pcat_sinf<Dual<T>>(Dual<T>((v + d) + vx, T(1)));
      const T w0 = v - E, w1 = (v + d) - E;
      const T i0 = g * u * a0.v * a0.v * w0, i1 = g * u * a1.v * a1.v * w1;
      const T slope = (i1 - i0) * T(1000.0);
      const T l_s = lr * (v - x1);  // adjoint of s, q's share included
      const T l_i1 = l_s * T(1000.0);
      const T l_i0 = -l_s * T(1000.0) - lr + lI;
      // d i / d (g, u, E) and d i / d (v + vx) at both voltages
      const T c0 = u * a0.v * a0.v, c1 = u * a1.v * a1.v;
      const T dw0 = g * u * T(2) * a0.v * a0.d * w0, dw1 = g * u * T(2) * a1.v * a1.d * w1;
      G.add(0, l_i0 * c0 * w0 + l_i1 * c1 * w1);
      G.add(1, l_i0 * dw0 + l_i1 * dw1);
      G.add(2, -(l_i0 * g * c0 + l_i1 * g * c1));
      lam[e.s[0]] += l_i0 * g * a0.v * a0.v * w0 + l_i1 * g * a1.v * a1.v * w1;
      lv += l_i0 * (dw0 + g * c0) + l_i1 * (dw1 + g * c1) + lr * slope;
      break;
    }
    default: {
      GateLayout gl = gate_layout(e.type);
      bool ca = e.type == CH_CAHVA || e.type == CH_CALVA;
      T g = P(0);
      T m = x[e.s[0]];
      T h = gl.g1 >= 0 ? x[e.s[1]] : T(1);
      T mp = ipow(m, gl.e0);
      T Gv = mp * h;
      T E = ca ? x[e.s[2]] : P(1);
      T lc, lE;
      ohmic(g * Gv, E, lc, lE);
      T dm = gl.e0 == 1 ? T(1) : T(gl.e0) * ipow(m, gl.e0 - 1);
      lam[e.s[0]] += g * dm * h * lc;
      if (gl.g1 >= 0) lam[e.s[1]] += g * mp * lc;
      G.add(0, Gv * lc);
      if (ca)
        lam[e.s[2]] += lE;
      else
        G.add(1, lE);
      break;
    }
  }
}

// d x'/d x and d x'/d v of one gate step at voltage v.
template <typename T>
__device__ __forceinline__ void gate_vjp(int g, T v, T x, T dt, T lx_new, T& lx_old, T& lv) {
  T e;
  Dual<T> xn = gate_step<Dual<T>, T>(g, Dual<T>(v, T(1)), x, dt, &e);
  lx_old = e * lx_new;
  lv += xn.d * lx_new;
}

// VJP of `channel_update` at the pre-update state `x` (the values this entry read).
// On entry lam holds the adjoint of the slots after the update; on return the adjoint
// of the slots before it.
template <typename T>
__device__ __forceinline__ void channel_update_vjp(const ChanEntry& e, const T* x, T* lam,
                                                   const Prm<T>& P, const PGradSink<T>& G, T v,
                                                   T dt, T& lv) {
  switch (e.type) {
    case CH_HH: {
      T lo;
      gate_vjp<T>(G_HH_M, v, x[e.s[0]], dt, lam[e.s[0]], lo, lv);
      lam[e.s[0]] = lo;
      gate_vjp<T>(G_HH_H, v, x[e.s[1]], dt, lam[e.s[1]], lo, lv);
      lam[e.s[1]] = lo;
      gate_vjp<T>(G_HH_N, v, x[e.s[2]], dt, lam[e.s[2]], lo, lv);
      lam[e.s[2]] = lo;
      break;
    }
    case CH_LEAK:
      break;
    case CH_SKE2: {
      T ez = T(1) + save_expm1(T(-1.0) / T(1.0) * dt);
      T lz = lam[e.s[0]];
      Dual<T> zi = ske2_zinf<Dual<T>>(Dual<T>(x[e.s[1]], T(1)));
      lam[e.s[0]] = ez * lz;
      lam[e.s[1]] += (T(1) - ez) * zi.d * lz;
      break;
    }
    case CH_CAPUMP: {
      T ica = x[e.cur];
      T cai = x[e.s[0]];
      T gamma = P(0), decay = P(1), depth = P(2), minCai = P(3);
      const T F2 = T(2) * T(96485);
      T drive = T(-10000.0) * ica * gamma / (F2 * depth);
      T cai_inf = minCai + decay * drive;
      T arg = -dt / decay;
      T em1 = save_expm1(arg);
      T ee = T(1) + em1;
      T lnew = lam[e.s[0]];
      T l_inf = -em1 * lnew;
      T l_ee = (cai - cai_inf) * lnew;
      T l_drive = decay * l_inf;
      lam[e.s[0]] = ee * lnew;
      if (e.cur >= 0) lam[e.cur] += T(-10000.0) * gamma / (F2 * depth) * l_drive;
      T l_decay = drive * l_inf + (arg > T(20) ? T(0) : l_ee * ee * dt / (decay * decay));
      G.add(0, T(-10000.0) * ica / (F2 * depth) * l_drive);
      G.add(1, l_decay);
      G.add(2, -drive / depth * l_drive);
      G.add(3, l_inf);
      break;
    }
    case CH_CANERNST: {
      T F = P(0), Tk = P(1), R = P(2);
      T C = R * Tk / (T(2) * F) * T(1000);
      T le = lam[e.s[0]];
      lam[e.s[0]] = T(0);
      lam[e.s[1]] += -C / x[e.s[1]] * le;
      lam[e.s[2]] += C / x[e.s[2]] * le;
      break;
    }
    case CH_PNA:
    case CH_PK:
    case CH_PCAT: {
      // gates of u = v - vt (Na, K) or v + vx (CaT): d/d vt = -d/du, d/d vx = d/du
      const bool cat = e.type == CH_PCAT;
      const int ps = cat ? 1 : 2;
      const T u = cat ? v + P(1) : v - P(2);
      const T sgn = cat ? T(1) : T(-1);
      GateLayout gl = gate_layout(e.type);
      T lo, lu = T(0);
      gate_vjp<T>(gl.g0, u, x[e.s[0]], dt, lam[e.s[0]], lo, lu);
      lam[e.s[0]] = lo;
      if (gl.g1 >= 0) {
        gate_vjp<T>(gl.g1, u, x[e.s[1]], dt, lam[e.s[1]], lo, lu);
        lam[e.s[1]] = lo;
      }
      lv += lu;
      G.add(ps, sgn * lu);
      break;
    }
    case CH_PKM: {
      T lo, lvk = T(0);
      const T taumax = P(1);
      const T pold = x[e.s[0]], ln = lam[e.s[0]];
      T ee;
      Dual<T> xn = gate_step<Dual<T>, T>(G_PKM_P, Dual<T>(v, T(1)), pold, dt, &ee,
                                         Dual<T>(T(1) / taumax));
      lo = ee * ln;
      lvk = xn.d * ln;
      // d x' / d taumax through the rate scale 1 / taumax
      Dual<T> xt = gate_step<Dual<T>, T>(G_PKM_P, Dual<T>(v), pold, dt, nullptr,
                                         Dual<T>(T(1) / taumax, -T(1) / (taumax * taumax)));
      lam[e.s[0]] = lo;
      lv += lvk;
      G.add(1, xt.d * ln);
      break;
    }
    default: {
      GateLayout gl = gate_layout(e.type);
      T lo;
      gate_vjp<T>(gl.g0, v, x[e.s[0]], dt, lam[e.s[0]], lo, lv);
      lam[e.s[0]] = lo;
      if (gl.g1 >= 0) {
        gate_vjp<T>(gl.g1, v, x[e.s[1]], dt, lam[e.s[1]], lo, lv);
        lam[e.s[1]] = lo;
      }
      break;
    }
  }
}

// Slots written by `channel_update` of an entry, for the undo log of the adjoint.
__device__ __forceinline__ int update_writes(const ChanEntry& e, short* out) {
  switch (e.type) {
    case CH_HH:
      out[0] = e.s[0]; out[1] = e.s[1]; out[2] = e.s[2];
      return 3;
    case CH_LEAK:
      return 0;
    case CH_SKE2:
    case CH_CAPUMP:
    case CH_CANERNST:
      out[0] = e.s[0];
      return 1;
    default: {
      GateLayout gl = gate_layout(e.type);
      out[0] = e.s[0];
      if (gl.g1 >= 0) { out[1] = e.s[1]; return 2; }
      return 1;
    }
  }
}

}  // namespace jxb

namespace jxb {

// Undo log of one node's channel updates for the adjoint: the slot, its value before
// the update, d new / d old and d new / d (v or the second input).
template <typename T, int N>
struct UndoLog {
  T old[N], dx[N], dy[N];
  short slot[N];
  int n = 0;
  __device__ __forceinline__ void push(short s, T o, T a, T b) {
    if (n < N) {
      slot[n] = s;
      old[n] = o;
      dx[n] = a;
      dy[n] = b;
      ++n;
    }
  }
};

// Gate step with its derivatives (dual number in v), logged.
template <typename T, int N>
__device__ __forceinline__ void gate_logged(int g, T v, T* x, short s, T dt, UndoLog<T, N>& L) {
  T e;
  Dual<T> xn = gate_step<Dual<T>, T>(g, Dual<T>(v, T(1)), x[s], dt, &e);
  L.push(s, x[s], e, xn.d);
  x[s] = xn.v;
}

// `channel_update` that logs every overwritten slot with the partial derivatives
// the reverse pass needs, so that the rate functions are evaluated once per step.
template <typename T, int N>
__device__ __forceinline__ void channel_update_logged(const ChanEntry& e, T* x, const Prm<T>& P,
                                                      T v, T dt, UndoLog<T, N>& L) {
  switch (e.type) {
    case CH_HH:
      gate_logged<T, N>(G_HH_M, v, x, e.s[0], dt, L);
      gate_logged<T, N>(G_HH_H, v, x, e.s[1], dt, L);
      gate_logged<T, N>(G_HH_N, v, x, e.s[2], dt, L);
      break;
    case CH_LEAK:
      break;
    case CH_SKE2: {
      const T em1 = save_expm1(T(-1.0) / T(1.0) * dt);
      Dual<T> zi = ske2_zinf<Dual<T>>(Dual<T>(x[e.s[1]], T(1)));
      const T z = x[e.s[0]];
      L.push(e.s[0], z, T(1) + em1, -em1 * zi.d);
      x[e.s[0]] = z + (z - zi.v) * em1;
      break;
    }
    case CH_CAPUMP:
    case CH_CANERNST:
    case CH_PKM:  // (its reverse pass recomputes the derivatives from the restored state)
      L.push(e.s[0], x[e.s[0]], T(0), T(0));
      channel_update<T>(e, x, P, v, dt);
      break;
    case CH_PNA:
    case CH_PK:
    case CH_PCAT: {  // gates of the shifted voltage; the log holds d x' / d u
      const T u = e.type == CH_PCAT ? v + P(1) : v - P(2);
      GateLayout gl = gate_layout(e.type);
      gate_logged<T, N>(gl.g0, u, x, e.s[0], dt, L);
      if (gl.g1 >= 0) gate_logged<T, N>(gl.g1, u, x, e.s[1], dt, L);
      break;
    }
    default: {
      GateLayout gl = gate_layout(e.type);
      gate_logged<T, N>(gl.g0, v, x, e.s[0], dt, L);
      if (gl.g1 >= 0) gate_logged<T, N>(gl.g1, v, x, e.s[1], dt, L);
      break;
    }
  }
}

// Reverse of `channel_update_logged`: restores the entry's slots from the log and
// applies its vector-Jacobian product.
template <typename T, int N>
__device__ __forceinline__ void channel_update_vjp_logged(const ChanEntry& e, T* x, T* lam,
                                                          const Prm<T>& P, const PGradSink<T>& G,
                                                          T v, T dt, T& lv, UndoLog<T, N>& L) {
  switch (e.type) {
    case CH_LEAK:
      break;
    case CH_SKE2: {
      --L.n;
      x[L.slot[L.n]] = L.old[L.n];
      const T lz = lam[e.s[0]];
      lam[e.s[0]] = L.dx[L.n] * lz;
      lam[e.s[1]] += L.dy[L.n] * lz;
      break;
    }
    case CH_CAPUMP:
    case CH_CANERNST:
    case CH_PKM:
      --L.n;
      x[L.slot[L.n]] = L.old[L.n];
      channel_update_vjp<T>(e, x, lam, P, G, v, dt, lv);
      break;
    case CH_PNA:
    case CH_PK:
    case CH_PCAT: {
      // as the default gates, with the shifted voltage's parameter: d/d vt = -d/du
      // (Na, K), d/d vx = d/du (CaT)
      const int ng = gate_layout(e.type).g1 >= 0 ? 2 : 1;
      T lu = T(0);
      for (int k = 0; k < ng; ++k) {
        --L.n;
        const short s = L.slot[L.n];
        x[s] = L.old[L.n];
        const T ln = lam[s];
        lam[s] = L.dx[L.n] * ln;
        lu += L.dy[L.n] * ln;
      }
      lv += lu;
      if (e.type == CH_PCAT)
        G.add(1, lu);
      else
        G.add(2, -lu);
      break;
    }
    default: {
      // Gates: pop in reverse order of the pushes.
      int ng = e.type == CH_HH ? 3 : (gate_layout(e.type).g1 >= 0 ? 2 : 1);
      for (int k = 0; k < ng; ++k) {
        --L.n;
        const short s = L.slot[L.n];
        x[s] = L.old[L.n];
        const T ln = lam[s];
        lam[s] = L.dx[L.n] * ln;
        lv += L.dy[L.n] * ln;
      }
      break;
    }
  }
}

}  // namespace jxb
