// Compile-time channel programs: the node classes whose channel list matches one of
// the programs below (and whose states are private to each channel, with no current
// slots) run this code instead of the generic interpreter of jxb_node.cuh. Slot and
// parameter offsets and gate ids are template constants, so there is no per-entry
// dispatch, and the adjoint keeps its undo log in registers (one stack frame per
// channel, unwound in reverse order). The arithmetic is the same as the generic path.
#pragma once
#include "jxb_node.cuh"

namespace jxb {

enum ProgramId { PROG_GENERIC = 0, PROG_HH = 1, PROG_L5PC_DEND = 2, PROG_L5PC_SOMA = 3 };

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

// The L5PC somatic channel set (mech/channels/l5pc.py) in insertion order: NaTs2T,
// SKv3_1, SKE2, CaNernstReversal, CaPump, CaHVA, CaLVA, Leak, with the reference's
// calcium coupling: SKE2 reads cai, the reversal is recomputed from cai before the
// pump integrates the previous step's i_Ca, CaHVA/CaLVA use the reversal and write
// i_Ca. Node-relative slots: 1-2 NaTs2T m,h; 3 SKv3_1 m; 4 SKE2 z; 5 cai; 6 eca;
// 7 cao; 8-9 CaHVA m,h; 10-11 CaLVA m,h; 12 i_Ca; parameters 0-16 in entry order
// (the lowering grants this program only to classes with exactly that layout). The
// operations and their order are the interpreter's (jxb_node.cuh: channel_update,
// channel_current, channel_current_vjp, channel_update_vjp and the logged replay),
// with constant slots and the undo values in registers.
template <typename T>
struct ProgL5pcSoma {
  static __device__ __forceinline__ T pump_target(const T* x, const T* p, T& drive) {
    drive = T(-10000.0) * x[12] * p[9] / (T(2) * T(96485) * p[11]);
    return p[12] + p[10] * drive;
  }
  static __device__ __forceinline__ T nernst_scale(const T* p) {  // R T / (2 F) in mV
    return p[8] * p[7] / (T(2) * p[6]) * T(1000);
  }

  static __device__ __forceinline__ void forward(T* x, const T* p, T dt, T& lin, T& cst) {
    const T v = x[0];
    x[1] = gate_step<T, T>(G_NATS2T_M, v, x[1], dt, nullptr);
    x[2] = gate_step<T, T>(G_NATS2T_H, v, x[2], dt, nullptr);
    x[3] = gate_step<T, T>(G_SKV31_M, v, x[3], dt, nullptr);
    {  // SKE2, tau_z = 1 (l5pc.py:488-500)
      const T zinf = ske2_zinf<T>(x[5]);
      const T em1 = save_expm1(T(-1.0) / T(1.0) * dt);
      const T z = x[4];
      x[4] = z + (z - zinf) * em1;
    }
    x[6] = nernst_scale(p) * lg(x[7] / x[5]);  // l5pc.py:891-902
    {  // CaPump (l5pc.py:842-861)
      const T cai = x[5];
      T drive;
      const T cai_inf = pump_target(x, p, drive);
      const T em1 = save_expm1(-dt / p[10]);
      x[5] = cai + (cai - cai_inf) * em1;
    }
    x[8] = gate_step<T, T>(G_CAHVA_M, v, x[8], dt, nullptr);
    x[9] = gate_step<T, T>(G_CAHVA_H, v, x[9], dt, nullptr);
    x[10] = gate_step<T, T>(G_CALVA_M, v, x[10], dt, nullptr);
    x[11] = gate_step<T, T>(G_CALVA_H, v, x[11], dt, nullptr);
    // Linearised currents at the updated state; i_Ca restarts from zero.
    x[12] = T(0);
    T slope = T(0), gge = T(0);
    {
      const T m = x[1];
      const T g = p[0] * ((m * m * m) * x[2]);
      slope += g;
      gge += g * p[1];
    }
    {
      const T g = p[2] * x[3];
      slope += g;
      gge += g * p[3];
    }
    {
      const T g = p[4] * x[4];
      slope += g;
      gge += g * p[5];
    }
    {
      const T m = x[8];
      const T g = p[13] * ((m * m) * x[9]);
      const T E = x[6];
      slope += g;
      gge += g * E;
      x[12] += g * (v - E);
    }
    {
      const T m = x[10];
      const T g = p[14] * ((m * m) * x[11]);
      const T E = x[6];
      slope += g;
      gge += g * E;
      x[12] += g * (v - E);
    }
    slope += p[15];
    gge += p[15] * p[16];
    lin = slope * T(1000.0);
    cst = gge * T(1000.0);
  }

  static __device__ __forceinline__ void adjoint(T* x, const T* p, T dt, AdjCtx<T>& c) {
    const T v = x[0];
    // Replay of the updates with the partial derivatives the reverse pass needs.
    T e1, e2, e3, e8, e9, e10, e11;
    const T o1 = x[1];
    const Dual<T> n1 = gate_step<Dual<T>, T>(G_NATS2T_M, Dual<T>(v, T(1)), o1, dt, &e1);
    x[1] = n1.v;
    const T o2 = x[2];
    const Dual<T> n2 = gate_step<Dual<T>, T>(G_NATS2T_H, Dual<T>(v, T(1)), o2, dt, &e2);
    x[2] = n2.v;
    const T o3 = x[3];
    const Dual<T> n3 = gate_step<Dual<T>, T>(G_SKV31_M, Dual<T>(v, T(1)), o3, dt, &e3);
    x[3] = n3.v;
    const T ske_em1 = save_expm1(T(-1.0) / T(1.0) * dt);
    const Dual<T> zi = ske2_zinf<Dual<T>>(Dual<T>(x[5], T(1)));
    const T o4 = x[4];
    const T dx4 = T(1) + ske_em1, dy4 = -ske_em1 * zi.d;
    x[4] = o4 + (o4 - zi.v) * ske_em1;
    const T o6 = x[6];
    const T C = nernst_scale(p);
    x[6] = C * lg(x[7] / x[5]);
    const T o5 = x[5];
    {
      T drive;
      const T cai_inf = pump_target(x, p, drive);
      const T em1 = save_expm1(-dt / p[10]);
      x[5] = o5 + (o5 - cai_inf) * em1;
    }
    const T o8 = x[8];
    const Dual<T> n8 = gate_step<Dual<T>, T>(G_CAHVA_M, Dual<T>(v, T(1)), o8, dt, &e8);
    x[8] = n8.v;
    const T o9 = x[9];
    const Dual<T> n9 = gate_step<Dual<T>, T>(G_CAHVA_H, Dual<T>(v, T(1)), o9, dt, &e9);
    x[9] = n9.v;
    const T o10 = x[10];
    const Dual<T> n10 = gate_step<Dual<T>, T>(G_CALVA_M, Dual<T>(v, T(1)), o10, dt, &e10);
    x[10] = n10.v;
    const T o11 = x[11];
    const Dual<T> n11 = gate_step<Dual<T>, T>(G_CALVA_H, Dual<T>(v, T(1)), o11, dt, &e11);
    x[11] = n11.v;

    // VJPs of the currents at the updated state, last channel first.
    const T lr = c.lr, x1 = c.x1;
    T* lam = c.lam;
    {  // Leak
      const T g = p[15], E = p[16];
      c.grad(15, lr * (E - x1));
      c.grad(16, g * lr);
    }
    const T lI = lam[12];
    {  // CaLVA
      const T g = p[14], m = x[10], h = x[11];
      const T mp = m * m, Gv = mp * h, E = x[6], cc = g * Gv;
      const T lc = lr * (E - x1) + (v - E) * lI;
      const T lE = cc * (lr - lI);
      c.lv += cc * lI;
      lam[10] += g * (T(2) * m) * h * lc;
      lam[11] += g * mp * lc;
      c.grad(14, Gv * lc);
      lam[6] += lE;
    }
    {  // CaHVA
      const T g = p[13], m = x[8], h = x[9];
      const T mp = m * m, Gv = mp * h, E = x[6], cc = g * Gv;
      const T lc = lr * (E - x1) + (v - E) * lI;
      const T lE = cc * (lr - lI);
      c.lv += cc * lI;
      lam[8] += g * (T(2) * m) * h * lc;
      lam[9] += g * mp * lc;
      c.grad(13, Gv * lc);
      lam[6] += lE;
    }
    {  // SKE2
      const T g = p[4], z = x[4], E = p[5];
      const T lc = lr * (E - x1);
      lam[4] += g * lc;
      c.grad(4, z * lc);
      c.grad(5, (g * z) * lr);
    }
    {  // SKv3_1
      const T g = p[2], m = x[3], E = p[3];
      const T lc = lr * (E - x1);
      lam[3] += g * lc;
      c.grad(2, m * lc);
      c.grad(3, (g * m) * lr);
    }
    {  // NaTs2T
      const T g = p[0], m = x[1], h = x[2];
      const T mp = m * m * m, Gv = mp * h, E = p[1];
      const T lc = lr * (E - x1);
      lam[1] += g * (T(3) * (m * m)) * h * lc;
      lam[2] += g * mp * lc;
      c.grad(0, Gv * lc);
      c.grad(1, (g * Gv) * lr);
    }
    // The step overwrote i_Ca: the adjoint of its previous value starts from zero.
    lam[12] = T(0);

    // VJPs of the updates, last channel first, restoring the state as it goes.
    auto gate_back = [&](int s, T old, T e, T d) {
      x[s] = old;
      const T ln = lam[s];
      lam[s] = e * ln;
      c.lv += d * ln;
    };
    gate_back(11, o11, e11, n11.d);
    gate_back(10, o10, e10, n10.d);
    gate_back(9, o9, e9, n9.d);
    gate_back(8, o8, e8, n8.d);
    x[5] = o5;
    {  // CaPump
      const T cai = x[5], ica = x[12];
      const T gamma = p[9], decay = p[10], depth = p[11];
      const T F2 = T(2) * T(96485);
      T drive;
      const T cai_inf = pump_target(x, p, drive);
      const T arg = -dt / decay;
      const T em1 = save_expm1(arg);
      const T ee = T(1) + em1;
      const T lnew = lam[5];
      const T l_inf = -em1 * lnew;
      const T l_ee = (cai - cai_inf) * lnew;
      const T l_drive = decay * l_inf;
      lam[5] = ee * lnew;
      lam[12] += T(-10000.0) * gamma / (F2 * depth) * l_drive;
      const T l_decay = drive * l_inf + (arg > T(20) ? T(0) : l_ee * ee * dt / (decay * decay));
      c.grad(9, T(-10000.0) * ica / (F2 * depth) * l_drive);
      c.grad(10, l_decay);
      c.grad(11, -drive / depth * l_drive);
      c.grad(12, l_inf);
    }
    x[6] = o6;
    {  // CaNernstReversal
      const T le = lam[6];
      lam[6] = T(0);
      lam[5] += -C / x[5] * le;
      lam[7] += C / x[7] * le;
    }
    x[4] = o4;
    {  // SKE2
      const T lz = lam[4];
      lam[4] = dx4 * lz;
      lam[5] += dy4 * lz;
    }
    gate_back(3, o3, e3, n3.d);
    gate_back(2, o2, e2, n2.d);
    gate_back(1, o1, e1, n1.d);
  }
};

template <typename T> using ProgL5pcDend = Program<T, CH_NATS2T, CH_SKV3_1, CH_M, CH_H, CH_LEAK>;

}  // namespace jxb
