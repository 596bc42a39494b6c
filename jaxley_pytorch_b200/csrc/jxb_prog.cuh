// Compile-time channel programs: the node classes whose channel list matches one of
// the programs below (and whose states are private to each channel, with no current
// slots) run this code instead of the generic interpreter of jxb_node.cuh. Slot and
// parameter offsets and gate ids are template constants, so there is no per-entry
// dispatch, and the adjoint keeps its undo log in registers (one stack frame per
// channel, unwound in reverse order). The arithmetic is the same as the generic path.
#pragma once
#include "jxb_node.cuh"

namespace jxb {

enum ProgramId { PROG_GENERIC = 0, PROG_HH = 1, PROG_L5PC_DEND = 2 };

// Layout of every channel type in a program: number of state and parameter slots.
template <int TYPE> struct ChanInfo;
template <> struct ChanInfo<CH_HH> { static constexpr int ns = 3, np = 6; };
template <> struct ChanInfo<CH_LEAK> { static constexpr int ns = 0, np = 2; };
template <> struct ChanInfo<CH_NATS2T> { static constexpr int ns = 2, np = 2; };
template <> struct ChanInfo<CH_SKV3_1> { static constexpr int ns = 1, np = 2; };
template <> struct ChanInfo<CH_M> { static constexpr int ns = 1, np = 2; };
template <> struct ChanInfo<CH_H> { static constexpr int ns = 1, np = 2; };

// Gate ids of the single- and two-gate channels of the programs.
template <int TYPE> struct Gates;
template <> struct Gates<CH_NATS2T> { static constexpr int g0 = G_NATS2T_M, g1 = G_NATS2T_H, e0 = 3; };
template <> struct Gates<CH_SKV3_1> { static constexpr int g0 = G_SKV31_M, g1 = -1, e0 = 1; };
template <> struct Gates<CH_M> { static constexpr int g0 = G_M_M, g1 = -1, e0 = 1; };
template <> struct Gates<CH_H> { static constexpr int g0 = G_H_M, g1 = -1, e0 = 1; };

// Context of one node for the adjoint.
template <typename T>
struct AdjCtx {
  T* lam;        // adjoint block of the node
  const T* pb;   // parameter bases of the node's run
  const int* gk; // gradient ranks of the node's run
  T* ga;         // gradient slots of the node
  T lr, x1;      // 1000 dt lambda_r / cm and the new voltage
  T lv;          // adjoint of the voltage before the step
  __device__ __forceinline__ void grad(int k, T g) {
    const int q = gk[k];
    if (q >= 0) ga[q] += g * pb[k];
  }
};

// ---- per channel code, slots S (first state) and P (first parameter) ----
template <typename T, int TYPE, int S, int P>
struct Chan {
  // Gated ohmic channel with g = P+0 and E = P+1 (NaTs2T, SKv3_1, M, H).
  using G = Gates<TYPE>;
  static __device__ __forceinline__ void update(T* x, const T*, T v, T dt) {
    x[S] = gate_step<T, T>(G::g0, v, x[S], dt, nullptr);
    if (G::g1 >= 0) x[S + 1] = gate_step<T, T>(G::g1, v, x[S + 1], dt, nullptr);
  }
  static __device__ __forceinline__ T cond(const T* x) {
    T m = x[S];
    T G0 = G::e0 == 3 ? m * m * m : m;
    return G::g1 >= 0 ? G0 * x[S + 1] : G0;
  }
  static __device__ __forceinline__ void current(const T* x, const T* p, T, T& slope, T& gge) {
    const T g = p[P] * cond(x);
    slope += g;
    gge += g * p[P + 1];
  }
  static __device__ __forceinline__ void current_vjp(const T* x, const T* p, T v, AdjCtx<T>& c) {
    const T Gc = cond(x);
    const T g = p[P] * Gc;
    const T E = p[P + 1];
    const T lc = c.lr * (E - c.x1);  // no current slot in a program
    c.grad(P, Gc * lc);
    c.grad(P + 1, g * c.lr);
    const T m = x[S];
    const T gm = p[P] * lc;
    if (G::g1 >= 0) {
      const T h = x[S + 1];
      const T mp = G::e0 == 3 ? m * m * m : m;
      const T dm = G::e0 == 3 ? T(3) * m * m : T(1);
      c.lam[S] += gm * dm * h;
      c.lam[S + 1] += gm * mp;
    } else {
      c.lam[S] += gm;
    }
    (void)v;
  }
  // Forward (logged in the caller's frame), then the rest of the program, then the
  // reverse of this channel.
  template <class Rest>
  static __device__ __forceinline__ void adjoint(T* x, const T* p, T v, T dt, AdjCtx<T>& c) {
    T e0, e1 = T(0);
    const T o0 = x[S];
    Dual<T> n0 = gate_step<Dual<T>, T>(G::g0, Dual<T>(v, T(1)), o0, dt, &e0);
    x[S] = n0.v;
    T o1 = T(0), d1 = T(0);
    if (G::g1 >= 0) {
      o1 = x[S + 1];
      Dual<T> n1 = gate_step<Dual<T>, T>(G::g1, Dual<T>(v, T(1)), o1, dt, &e1);
      x[S + 1] = n1.v;
      d1 = n1.d;
    }
    Rest::adjoint(x, p, v, dt, c);
    if (G::g1 >= 0) {
      x[S + 1] = o1;
      const T l1 = c.lam[S + 1];
      c.lam[S + 1] = e1 * l1;
      c.lv += d1 * l1;
    }
    x[S] = o0;
    const T l0 = c.lam[S];
    c.lam[S] = e0 * l0;
    c.lv += n0.d * l0;
  }
};

template <typename T, int S, int P>
struct Chan<T, CH_LEAK, S, P> {  // channels/pospischil.py:64-68
  static __device__ __forceinline__ void update(T*, const T*, T, T) {}
  static __device__ __forceinline__ void current(const T*, const T* p, T, T& slope, T& gge) {
    slope += p[P];
    gge += p[P] * p[P + 1];
  }
  static __device__ __forceinline__ void current_vjp(const T*, const T* p, T, AdjCtx<T>& c) {
    const T lc = c.lr * (p[P + 1] - c.x1);
    c.grad(P, lc);
    c.grad(P + 1, p[P] * c.lr);
  }
  template <class Rest>
  static __device__ __forceinline__ void adjoint(T* x, const T* p, T v, T dt, AdjCtx<T>& c) {
    Rest::adjoint(x, p, v, dt, c);
  }
};

template <typename T, int S, int P>
struct Chan<T, CH_HH, S, P> {  // channels/hh.py:37-67
  static __device__ __forceinline__ void update(T* x, const T*, T v, T dt) {
    x[S] = gate_step<T, T>(G_HH_M, v, x[S], dt, nullptr);
    x[S + 1] = gate_step<T, T>(G_HH_H, v, x[S + 1], dt, nullptr);
    x[S + 2] = gate_step<T, T>(G_HH_N, v, x[S + 2], dt, nullptr);
  }
  static __device__ __forceinline__ void current(const T* x, const T* p, T, T& slope, T& gge) {
    const T m = x[S], h = x[S + 1], n = x[S + 2];
    const T gNa = p[P] * (m * m * m) * h, gK = p[P + 1] * (n * n * n * n), gL = p[P + 2];
    slope += gNa + gK + gL;
    gge += gNa * p[P + 3] + gK * p[P + 4] + gL * p[P + 5];
  }
  static __device__ __forceinline__ void current_vjp(const T* x, const T* p, T, AdjCtx<T>& c) {
    const T m = x[S], h = x[S + 1], n = x[S + 2];
    const T G1 = (m * m * m) * h, G2 = n * n * n * n;
    const T l1 = c.lr * (p[P + 3] - c.x1), l2 = c.lr * (p[P + 4] - c.x1), l3 = c.lr * (p[P + 5] - c.x1);
    c.lam[S] += p[P] * T(3) * m * m * h * l1;
    c.lam[S + 1] += p[P] * m * m * m * l1;
    c.lam[S + 2] += p[P + 1] * T(4) * n * n * n * l2;
    c.grad(P, G1 * l1);
    c.grad(P + 1, G2 * l2);
    c.grad(P + 2, l3);
    c.grad(P + 3, p[P] * G1 * c.lr);
    c.grad(P + 4, p[P + 1] * G2 * c.lr);
    c.grad(P + 5, p[P + 2] * c.lr);
  }
  template <class Rest>
  static __device__ __forceinline__ void adjoint(T* x, const T* p, T v, T dt, AdjCtx<T>& c) {
    T e[3];
    T o[3];
    T d[3];
    const int g[3] = {G_HH_M, G_HH_H, G_HH_N};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      o[k] = x[S + k];
      Dual<T> nk = gate_step<Dual<T>, T>(g[k], Dual<T>(v, T(1)), o[k], dt, &e[k]);
      x[S + k] = nk.v;
      d[k] = nk.d;
    }
    Rest::adjoint(x, p, v, dt, c);
#pragma unroll
    for (int k = 2; k >= 0; --k) {
      x[S + k] = o[k];
      const T l = c.lam[S + k];
      c.lam[S + k] = e[k] * l;
      c.lv += d[k] * l;
    }
  }
};

// ---- a program: channels in insertion order, consecutive slots from 1 (slot 0 = v)
// and consecutive parameters from 0 ----
template <typename T, int S, int P, int... TYPES>
struct Prog;

template <typename T, int S, int P>
struct Prog<T, S, P> {
  static __device__ __forceinline__ void update(T*, const T*, T, T) {}
  static __device__ __forceinline__ void current(const T*, const T*, T, T&, T&) {}
  static __device__ __forceinline__ void current_vjp(const T*, const T*, T, AdjCtx<T>&) {}
};

template <typename T, int S, int P, int T1, int... TS>
struct Prog<T, S, P, T1, TS...> {
  using Head = Chan<T, T1, S, P>;
  using Rest = Prog<T, S + ChanInfo<T1>::ns, P + ChanInfo<T1>::np, TS...>;
  static __device__ __forceinline__ void update(T* x, const T* p, T v, T dt) {
    Head::update(x, p, v, dt);
    Rest::update(x, p, v, dt);
  }
  static __device__ __forceinline__ void current(const T* x, const T* p, T v, T& s, T& g) {
    Head::current(x, p, v, s, g);
    Rest::current(x, p, v, s, g);
  }
  static __device__ __forceinline__ void current_vjp(const T* x, const T* p, T v, AdjCtx<T>& c) {
    Rest::current_vjp(x, p, v, c);
    Head::current_vjp(x, p, v, c);
  }
};

// Nested adjoint: channel k's frame holds its undo values while the channels after
// it run; the innermost frame applies the VJP of all currents.
template <class Full, typename T, int S, int P, int... TYPES>
struct ProgAdj;

template <class Full, typename T, int S, int P>
struct ProgAdj<Full, T, S, P> {
  static __device__ __forceinline__ void adjoint(T* x, const T* p, T v, T, AdjCtx<T>& c) {
    Full::current_vjp(x, p, v, c);
  }
};

template <class Full, typename T, int S, int P, int T1, int... TS>
struct ProgAdj<Full, T, S, P, T1, TS...> {
  using Rest = ProgAdj<Full, T, S + ChanInfo<T1>::ns, P + ChanInfo<T1>::np, TS...>;
  static __device__ __forceinline__ void adjoint(T* x, const T* p, T v, T dt, AdjCtx<T>& c) {
    Chan<T, T1, S, P>::template adjoint<Rest>(x, p, v, dt, c);
  }
};

template <typename T, int... TYPES>
struct Program {
  using F = Prog<T, 1, 0, TYPES...>;
  using A = ProgAdj<F, T, 1, 0, TYPES...>;
  // Forward: updates then linearised currents (uA/cm^2).
  static __device__ __forceinline__ void forward(T* x, const T* p, T dt, T& lin, T& cst) {
    const T v = x[0];
    F::update(x, p, v, dt);
    T slope = T(0), gge = T(0);
    F::current(x, p, v, slope, gge);
    lin = slope * T(1000.0);
    cst = gge * T(1000.0);
  }
  static __device__ __forceinline__ void adjoint(T* x, const T* p, T dt, AdjCtx<T>& c) {
    A::adjoint(x, p, x[0], dt, c);
  }
};

template <typename T> using ProgHH = Program<T, CH_HH>;
template <typename T> using ProgL5pcDend = Program<T, CH_NATS2T, CH_SKV3_1, CH_M, CH_H, CH_LEAK>;

}  // namespace jxb
