// Fixed in-degree synapse step (KineticSynapse, SigmoidRateSynapse) in the regular
// layout: E = T * k synapses ordered by postsynaptic target, k per target
// (jaxley-pytorch kernels/synapse_step.py, modules/network.py:381-478).
//
// Lane groups: L lanes (a power of two, about 16 synapses each) serve one
// (row, target) pair; lane c takes the target's synapses c, c + L, c + 2L, ..., so
// that the 32 / L groups of a warp read L consecutive values of each state and
// parameter array per instruction (whole 32-byte sectors at L = 8), sum their
// synapses in registers and combine them with log2(L) shuffles. No shared-memory
// reductions and no block barriers in the forward.
//
// forward:  32 / L targets per warp, 4 rows per warp (the synapse constants loaded
//           once for them), 4 warps per CTA over further rows.
// backward: one CTA per group of 32 / L targets (two for k up to 128, one above)
//           with 8 warps over the batch rows (each warp kRowsPerWarp rows per
//           pass). Per synapse chunk (one value of i in c + i L) the parameter
//           gradients are summed over the warp's rows in registers and over the
//           warps in shared memory in a fixed order, and the presynaptic voltage
//           gradients of the chunk are staged in shared memory and written to an
//           (E, batch) buffer row-contiguously; a second kernel sums them per
//           presynaptic node through the transposed index (four warps per node,
//           each over a quarter of its synapses). No atomics, deterministic.
// float: fast reciprocal / division / exp (jxb_math.cuh); float64 stays exact.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "jxb.h"
#include "jxb_math.cuh"

namespace jxb {
extern thread_local char g_err[512];
void set_err(const char* what, cudaError_t e);
}  // namespace jxb

namespace {

using namespace jxb;

template <typename T> __device__ __forceinline__ T qdiv(T x, T y) { return jxb::fdiv(x, y); }
template <typename T> __device__ __forceinline__ T sigm(T x) { return jxb::rcp(T(1) + ex(-x)); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
struct SynP {
  const T* p[6];
};

// One synapse's constants: parameters in the reference order (Kinetic: gS, e_syn,
// alpha, beta, v_th, delta; SigmoidRate: gS, x_offset, slope), the area of its
// target compartment and its presynaptic node.
template <typename T>
struct SynC {
  T gs, ar, q1, q2, q3, q4, q5;
  int pre;
};

// Read-only loads through the non-coherent path: the arrays a launch reads are never
// written by it, which also lets the compiler issue the loads of several synapses
// before their arithmetic.
template <typename T>
__device__ __forceinline__ T rd(const T* p) { return __ldg(p); }

template <typename T>
__device__ __forceinline__ SynC<T> load_syn(const JxbSynArgs& a, const SynP<T>& P, int64_t e) {
  SynC<T> c;
  c.pre = rd(a.pre + e);
  c.gs = rd(P.p[0] + e);
  c.ar = rd((const T*)a.area + e);
  c.q1 = rd(P.p[1] + e);
  c.q2 = rd(P.p[2] + e);
  c.q3 = a.model == 0 ? rd(P.p[3] + e) : T(0);
  c.q4 = a.model == 0 ? rd(P.p[4] + e) : T(0);
  c.q5 = a.model == 0 ? rd(P.p[5] + e) : T(1);
  return c;
}

// Forward of one synapse and row (synapses/kinetic.py:37-63, sigmoid_rate.py:43-50):
// the new kinetic state, the current i0 at vp, and the synapse's terms of the
// target's slope and offset in uA/cm^2 (kernels/synapse_step.py:150-180 take them as
// the finite difference of the current over `diff` and its value less slope x vp).
// The kinetic current gS s (v - e_syn) is linear in v: its slope is exactly
// gS s 1e5 / area and its offset -slope e_syn, which is what the finite difference
// evaluates to up to rounding (here without the float32 cancellation of a 1e-3 mV
// difference of two currents of tens of mV). The rate synapse keeps the reference's
// difference quotient.
template <typename T>
__device__ __forceinline__ void syn_forward_one(int model, const SynC<T>& c, T s, T vpre, T vp, T dt, T diff,
                                                T& s_new, T& i0, T& lin_t, T& cst_t) {
  if (model == 0) {
    const T tr = sigm(qdiv<T>(vpre - c.q4, c.q5));
    const T aa = c.q2 * tr;
    const T rate = aa + c.q3;
    const T s_inf = qdiv<T>(aa, rate);
    s_new = s_inf + (s - s_inf) * ex(-dt * rate);
    const T gsn = c.gs * s_new;
    i0 = gsn * (vp - c.q1);
    lin_t = qdiv<T>(gsn, c.ar) * T(100000.0);
    cst_t = -lin_t * c.q1;
  } else {
    s_new = T(0);
    i0 = -c.gs * sigm((vpre - c.q1) * c.q2);
    const T i1 = -c.gs * sigm(((vpre + diff) - c.q1) * c.q2);
    const T d0 = qdiv<T>(i0, c.ar) * T(100000.0);
    const T d1 = qdiv<T>(i1, c.ar) * T(100000.0);
    lin_t = qdiv<T>(d1 - d0, diff);
    cst_t = d0 - lin_t * vp;
  }
}

// Adjoint of one synapse and row (kernels/synapse_step.py:256-305) given the
// gradients of the target's slope and offset (glin, gconst), of the new state and of
// the current: adds the parameter gradients to gp[], returns the state gradient in
// g_s, the target-voltage gradient in g_vp and the presynaptic one in g_vpre.
template <typename T>
__device__ __forceinline__ void syn_backward_one(int model, const SynC<T>& c, T s, T vpre, T vp, T dt, T diff,
                                                 T glin, T gconst, T g_sn_in, T g_cur, T (&gp)[6], T& g_s,
                                                 T& g_vp, T& g_vpre) {
  if (model == 0) {
    // slope K gS s_new and offset -K gS s_new e_syn (K = 1e5 / area), current
    // gS s_new (vp - e_syn): the target voltage enters through the current only.
    const T x = qdiv<T>(vpre - c.q4, c.q5);
    const T tr = sigm(x);
    const T aa = c.q2 * tr;
    const T rate = aa + c.q3;
    const T s_inf = qdiv<T>(aa, rate);
    const T decay = ex(-dt * rate);
    const T s_new = s_inf + (s - s_inf) * decay;
    const T K = qdiv<T>(T(100000.0), c.ar);
    const T w0 = vp - c.q1;
    const T g_c = (glin - gconst * c.q1) * K + g_cur * w0;  // d loss / d (gS s_new)
    const T g_sn = c.gs * g_c + g_sn_in;
    g_vp = g_cur * c.gs * s_new;
    const T g_sinf = g_sn * (T(1) - decay);
    const T g_rate = -dt * decay * g_sn * (s - s_inf) - qdiv<T>(g_sinf * s_inf, rate);
    const T g_a = qdiv<T>(g_sinf, rate) + g_rate;
    const T g_x = g_a * c.q2 * tr * (T(1) - tr);
    g_vpre = qdiv<T>(g_x, c.q5);
    g_s = g_sn * decay;
    gp[0] += s_new * g_c;
    gp[1] += -c.gs * s_new * (gconst * K + g_cur);
    gp[2] += g_a * tr;
    gp[3] += g_rate;
    gp[4] += -g_vpre;
    gp[5] += -g_vpre * x;
  } else {
    const T u0 = vpre - c.q1;
    const T u1 = (vpre + diff) - c.q1;
    const T sig0 = sigm(u0 * c.q2);
    const T sig1 = sigm(u1 * c.q2);
    const T i0 = -c.gs * sig0;
    const T i1 = -c.gs * sig1;
    const T d0 = qdiv<T>(i0, c.ar) * T(100000.0);
    const T d1 = qdiv<T>(i1, c.ar) * T(100000.0);
    const T vt = qdiv<T>(d1 - d0, diff);
    const T g_vt = glin - gconst * vp;
    g_vp = -gconst * vt;
    const T g_d1 = qdiv<T>(g_vt, diff);
    const T g_d0 = gconst - g_d1;
    const T g_i0 = qdiv<T>(g_d0 * T(100000.0), c.ar) + g_cur;
    const T g_i1 = qdiv<T>(g_d1 * T(100000.0), c.ar);
    const T g_z0 = -c.gs * g_i0 * sig0 * (T(1) - sig0);
    const T g_z1 = -c.gs * g_i1 * sig1 * (T(1) - sig1);
    g_vpre = (g_z0 + g_z1) * c.q2;
    g_s = T(0);
    gp[0] += -(g_i0 * sig0 + g_i1 * sig1);
    gp[1] += -g_vpre;
    gp[2] += g_z0 * u0 + g_z1 * u1;
  }
}

// Sum over the L lanes of a group (aligned groups of L consecutive lanes).
template <int L, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kFwdWarps = 4;      // warps per forward CTA
constexpr int kFwdRows = 4;       // batch rows of a forward warp
constexpr int kFwdBatch = 2;      // synapses of a lane loaded together in the forward
constexpr int kBwdWarps = 8;      // warps per backward CTA
constexpr int kRowsPerWarp = 4;   // rows of a backward warp per pass

// float: at most 64 registers, so that eight CTAs (32 warps) per SM keep more gathers
// in flight than wider batches of loads per thread with fewer warps would.
template <typename T, int L>
__global__ void __launch_bounds__(32 * kFwdWarps, sizeof(T) == 4 ? 8 : 4) syn_forward_kernel(JxbSynArgs a, SynP<T> P) {
  constexpr int TPW = 32 / L;  // targets per warp
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = lane & (L - 1);
  const int nt = a.n_syn / a.k;
  const int tgt = blockIdx.x * TPW + lane / L;
  // the warp's rows: b0, b0 + 1, ..., b0 + kFwdRows - 1 (the synapse constants are
  // loaded once for all of them)
  const int64_t b0 = ((int64_t)blockIdx.y * kFwdWarps + warp) * kFwdRows;
  const bool ok = tgt < nt && b0 < a.batch;
  const int nr = ok ? (int)min((int64_t)kFwdRows, (int64_t)a.batch - b0) : 0;
  const T* sc = (const T*)a.scalars;
  const T dt = sc[0], diff = sc[1];
  T lin[kFwdRows], cst[kFwdRows], vp[kFwdRows];
  const int node = ok ? (a.targets_are_nodes ? tgt : a.targets[tgt]) : 0;
#pragma unroll
  for (int r = 0; r < kFwdRows; ++r) {
    lin[r] = cst[r] = T(0);
    vp[r] = r < nr ? rd((const T*)a.v + (b0 + r) * a.n_nodes + node) : T(0);
  }
  if (ok) {
    // kFwdBatch synapses of the lane at a time: their constants (indices clamped to
    // the target's range), then per row the states and presynaptic voltages of all
    // of them, then the arithmetic, so that a warp keeps many independent loads in
    // flight.
    for (int kb = c; kb < a.k; kb += kFwdBatch * L) {
      SynC<T> y[kFwdBatch];
      int64_t e[kFwdBatch];
#pragma unroll
      for (int u = 0; u < kFwdBatch; ++u) {
        e[u] = (int64_t)tgt * a.k + min(kb + u * L, a.k - 1);
        y[u] = load_syn<T>(a, P, e[u]);
      }
#pragma unroll
      for (int r = 0; r < kFwdRows; ++r) {
        if (r >= nr) break;
        const int64_t b = b0 + r;
        const T* v = (const T*)a.v + b * a.n_nodes;
        const T* s_row = a.model == 0 ? (const T*)a.s + b * a.n_syn : nullptr;
        T* sn_row = a.model == 0 ? (T*)a.s_new + b * a.n_syn : nullptr;
        T sv[kFwdBatch], vv[kFwdBatch];
#pragma unroll
        for (int u = 0; u < kFwdBatch; ++u) {
          sv[u] = s_row ? rd(s_row + e[u]) : T(0);
          vv[u] = rd(v + y[u].pre);
        }
#pragma unroll
        for (int u = 0; u < kFwdBatch; ++u) {
          if (kb + u * L >= a.k) break;
          T s_new, i0, lt, ct;
          syn_forward_one<T>(a.model, y[u], sv[u], vv[u], vp[r], dt, diff, s_new, i0, lt, ct);
          if (sn_row) sn_row[e[u]] = s_new;
          if (a.store_current) ((T*)a.current)[b * a.n_syn + e[u]] = i0;
          lin[r] += lt;
          cst[r] += ct;
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kFwdRows; ++r) {
    const T l = group_sum<L>(lin[r]);
    const T q = group_sum<L>(cst[r]);
    if (c == 0 && r < nr) {
      ((T*)a.lin)[(b0 + r) * nt + tgt] = l;
      ((T*)a.cst)[(b0 + r) * nt + tgt] = q;
    }
  }
}

template <typename T, int L>
__global__ void __launch_bounds__(32 * kBwdWarps) syn_backward_kernel(JxbSynArgs a, SynP<T> P) {
  constexpr int TPW = 32 / L;
  constexpr int RP = kBwdWarps * kRowsPerWarp;  // rows per pass
  // red[warp][lane][param]: the warps' parameter gradients of a chunk;
  // tile[lane][row of the pass]: its presynaptic voltage gradients. Two of each,
  // alternating by chunk: a chunk's sums and stores read one pair while the next
  // chunk's arithmetic fills the other, so one barrier per chunk separates them.
  __shared__ T red_buf[2][kBwdWarps * 32 * 6];
  __shared__ T tile_buf[2][32 * RP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = lane & (L - 1);
  const int nt = a.n_syn / a.k;
  const int tgt = blockIdx.x * TPW + lane / L;
  const bool tok = tgt < nt;
  const T* sc = (const T*)a.scalars;
  const T dt = sc[0], diff = sc[1];
  const int node = tok ? (a.targets_are_nodes ? tgt : a.targets[tgt]) : 0;
  const int np = a.model == 0 ? 6 : 3;
  int need_rows = 0;
  for (int q = 0; q < np; ++q) need_rows += (a.need >> q) & 1;
  T* g_pre = (T*)a.g_pre;
  const int J = (a.k + L - 1) / L;  // synapse chunks
  for (int b0 = 0; b0 < a.batch; b0 += RP) {  // passes over the rows
    const int nr = min(RP, a.batch - b0);
    T gvp[kRowsPerWarp];
    T glin[kRowsPerWarp], gconst[kRowsPerWarp], vp[kRowsPerWarp];
#pragma unroll
    for (int m = 0; m < kRowsPerWarp; ++m) {
      gvp[m] = T(0);
      const int r = m * kBwdWarps + warp;
      const int64_t b = b0 + r;
      const bool row = tok && r < nr;
      glin[m] = row ? rd((const T*)a.g_lin + b * nt + tgt) : T(0);
      gconst[m] = row ? rd((const T*)a.g_const + b * nt + tgt) : T(0);
      vp[m] = row ? rd((const T*)a.v + b * a.n_nodes + node) : T(0);
    }
    // The next chunk's synapse constants are loaded while the current chunk computes.
    SynC<T> y_next = load_syn<T>(a, P, (int64_t)(tok ? tgt : 0) * a.k + ((tok && c < a.k) ? c : 0));
    for (int i = 0; i < J; ++i) {
      T* const red = red_buf[i & 1];
      T* const tile = tile_buf[i & 1];
      const int kk = i * L + c;
      const bool act = tok && kk < a.k;
      const int64_t e = (int64_t)(tok ? tgt : 0) * a.k + (act ? kk : 0);
      const SynC<T> y = y_next;
      if (i + 1 < J) {
        const int k1 = kk + L;
        y_next = load_syn<T>(a, P, (int64_t)(tok ? tgt : 0) * a.k + ((tok && k1 < a.k) ? k1 : 0));
      }
      T gp[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
#pragma unroll
      for (int m = 0; m < kRowsPerWarp; ++m) {
        const int r = m * kBwdWarps + warp;
        T g_vpre = T(0);
        if (act && r < nr) {
          const int64_t b = b0 + r;
          const T* v = (const T*)a.v + b * a.n_nodes;
          const T s = a.model == 0 ? rd((const T*)a.s + b * a.n_syn + e) : T(0);
          const T gsn = a.g_s_new ? rd((const T*)a.g_s_new + b * a.n_syn + e) : T(0);
          const T gcu = a.g_current ? rd((const T*)a.g_current + b * a.n_syn + e) : T(0);
          T g_s, g_vp;
          syn_backward_one<T>(a.model, y, s, rd(v + y.pre), vp[m], dt, diff, glin[m], gconst[m], gsn, gcu, gp,
                              g_s, g_vp, g_vpre);
          if (a.model == 0) ((T*)a.g_s)[b * a.n_syn + e] = g_s;
          gvp[m] += g_vp;
        }
        tile[lane * RP + r] = g_vpre;
      }
#pragma unroll
      for (int q = 0; q < 6; ++q) red[(warp * 32 + lane) * 6 + q] = gp[q];
      __syncthreads();
      // Parameter gradients of the chunk's synapses: summed over the warps in order.
      for (int w = threadIdx.x; w < 32 * need_rows; w += blockDim.x) {
        const int ln = w & 31, qi = w >> 5;
        int q = 0, seen = -1;
        for (; q < np; ++q)
          if (((a.need >> q) & 1) && ++seen == qi) break;
        const int t2 = blockIdx.x * TPW + ln / L, k2 = i * L + (ln & (L - 1));
        if (t2 < nt && k2 < a.k) {
          T acc = T(0);
          for (int ww = 0; ww < kBwdWarps; ++ww) acc += red[(ww * 32 + ln) * 6 + q];
          T& out = ((T*)a.g_params)[(int64_t)qi * a.n_syn + (int64_t)t2 * a.k + k2];
          out = (a.accumulate || b0 > 0) ? out + acc : acc;
        }
      }
      // Presynaptic voltage gradients of the chunk, row-contiguous per synapse (a
      // warp writes one synapse's rows of the pass).
      static_assert(RP == 32, "one warp per synapse row of the tile");
      for (int w = threadIdx.x; w < 32 * 32; w += blockDim.x) {
        const int ln = w >> 5, r = w & 31;
        const int t2 = blockIdx.x * TPW + ln / L, k2 = i * L + (ln & (L - 1));
        if (r < nr && t2 < nt && k2 < a.k) g_pre[((int64_t)t2 * a.k + k2) * a.batch + b0 + r] = tile[ln * RP + r];
      }
    }
    __syncthreads();  // the last chunks' buffers are read before the next pass writes them
    // The target-voltage gradient of every (row, target): added to g_v here when
    // accumulating (one lane group owns the pair), else by syn_post_kernel.
#pragma unroll
    for (int m = 0; m < kRowsPerWarp; ++m) {
      const T g = group_sum<L>(gvp[m]);
      const int r = m * kBwdWarps + warp;
      if (tok && c == 0 && r < nr) {
        const int64_t b = b0 + r;
        if (a.accumulate) ((T*)a.g_v)[b * a.n_nodes + node] += g;
        else ((T*)a.g_post)[b * nt + tgt] = g;
      }
    }
  }
}

// g_v[b, pre_nodes[j]] = sum over the synapses of node j of g_pre[e, b]; then the
// postsynaptic terms g_post[b, t] are added at the targets.
constexpr int kPresumParts = 4;  // warps per presynaptic node, each summing a quarter of its synapses

// g_v[b, pre_nodes[j]] = sum over the synapses e of node j of g_pre[e, b]: one CTA per
// (node, 32 rows), warp p sums the entries p, p + 4, ... of the node's list for its
// lane's row (coalesced rows of g_pre), the four partial sums are added in order.
template <typename T>
__global__ void __launch_bounds__(32 * kPresumParts) syn_presum_kernel(JxbSynArgs a) {
  __shared__ T part[kPresumParts][32];
  const int j = blockIdx.x;
  const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
  const int64_t b = (int64_t)blockIdx.y * 32 + lane;
  const bool ok = b < a.batch;
  const T* g_pre = (const T*)a.g_pre;
  const int* inv = a.inv + (int64_t)j * a.inv_width;
  T acc = T(0);
  constexpr int U = 8;  // entries loaded together
  for (int q0 = p; q0 < a.inv_width; q0 += U * kPresumParts) {
    int e[U];
    T g[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = q0 + u * kPresumParts;
      e[u] = q < a.inv_width ? rd(inv + q) : -1;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) g[u] = (ok && e[u] >= 0) ? rd(g_pre + (int64_t)e[u] * a.batch + b) : T(0);
#pragma unroll
    for (int u = 0; u < U; ++u) acc += g[u];
  }
  part[p][lane] = acc;
  __syncthreads();
  if (p == 0 && ok) {
    T sum = part[0][lane];
#pragma unroll
    for (int w = 1; w < kPresumParts; ++w) sum += part[w][lane];
    T& out = ((T*)a.g_v)[b * a.n_nodes + a.pre_nodes[j]];
    out = a.accumulate ? out + sum : sum;
  }
}

template <typename T>
__global__ void syn_post_kernel(JxbSynArgs a) {
  const int nt = a.n_syn / a.k;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)nt * a.batch) return;
  const int t = idx % nt;
  const int64_t b = idx / nt;
  const int node = a.targets_are_nodes ? t : a.targets[t];
  ((T*)a.g_v)[b * a.n_nodes + node] += ((const T*)a.g_post)[b * nt + t];
}

// Lanes per (row, target): a power of two giving about 16 synapses per lane.
inline int syn_lanes(int k) {
  int L = 1;
  while (L < 32 && L * 16 < k) L *= 2;
  return L;
}

template <typename T>
int fwd(const JxbSynArgs& a, cudaStream_t st) {
  SynP<T> P;
  for (int q = 0; q < 6; ++q) P.p[q] = (const T*)a.p[q];
  const int nt = a.n_syn / a.k;
  const int L = syn_lanes(a.k);
  const int rows_per_cta = kFwdWarps * kFwdRows;
  const dim3 grid((unsigned)((nt + 32 / L - 1) / (32 / L)), (unsigned)((a.batch + rows_per_cta - 1) / rows_per_cta));
  const int th = 32 * kFwdWarps;
  switch (L) {
    case 1: syn_forward_kernel<T, 1><<<grid, th, 0, st>>>(a, P); break;
    case 2: syn_forward_kernel<T, 2><<<grid, th, 0, st>>>(a, P); break;
    case 4: syn_forward_kernel<T, 4><<<grid, th, 0, st>>>(a, P); break;
    case 8: syn_forward_kernel<T, 8><<<grid, th, 0, st>>>(a, P); break;
    case 16: syn_forward_kernel<T, 16><<<grid, th, 0, st>>>(a, P); break;
    default: syn_forward_kernel<T, 32><<<grid, th, 0, st>>>(a, P); break;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("syn_forward_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

template <typename T>
int bwd(const JxbSynArgs& a, cudaStream_t st) {
  SynP<T> P;
  for (int q = 0; q < 6; ++q) P.p[q] = (const T*)a.p[q];
  const int nt = a.n_syn / a.k;
  cudaError_t e = cudaSuccess;
  if (!a.accumulate) {  // the op's g_v: zero where neither sum writes
    e = cudaMemsetAsync(a.g_v, 0, sizeof(T) * (size_t)a.batch * a.n_nodes, st);
    if (e != cudaSuccess) {
      set_err("cudaMemsetAsync", e);
      return JXB_ERR_LAUNCH;
    }
  }
  // Two targets per CTA (L = 16) for up to 128 synapses a target, one (L = 32) above:
  // more CTAs than the forward's lane groups keep more warps in flight (measured at
  // 1024 and 2048 targets x 100 synapses x 32 rows against L = 32: 2 and 9 % faster).
  const int L = a.k > 128 ? 32 : (a.k > 32 ? 16 : syn_lanes(a.k));
  const unsigned grid = (unsigned)((nt + 32 / L - 1) / (32 / L));
  const int th = 32 * kBwdWarps;
  switch (L) {
    case 1: syn_backward_kernel<T, 1><<<grid, th, 0, st>>>(a, P); break;
    case 2: syn_backward_kernel<T, 2><<<grid, th, 0, st>>>(a, P); break;
    case 4: syn_backward_kernel<T, 4><<<grid, th, 0, st>>>(a, P); break;
    case 8: syn_backward_kernel<T, 8><<<grid, th, 0, st>>>(a, P); break;
    case 16: syn_backward_kernel<T, 16><<<grid, th, 0, st>>>(a, P); break;
    default: syn_backward_kernel<T, 32><<<grid, th, 0, st>>>(a, P); break;
  }
  const int threads = 256;
  const int64_t n1 = (int64_t)a.n_pre_nodes * a.batch;
  if (n1 > 0)
    syn_presum_kernel<T><<<dim3((unsigned)a.n_pre_nodes, (unsigned)((a.batch + 31) / 32)), 32 * kPresumParts, 0, st>>>(a);
  const int64_t n2 = (int64_t)nt * a.batch;
  if (!a.accumulate) syn_post_kernel<T><<<(unsigned)((n2 + threads - 1) / threads), threads, 0, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("syn_backward_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

int check(const JxbSynArgs* a, bool backward) {
  if (!a || a->k <= 0 || a->n_syn % a->k != 0 || a->batch <= 0 || !a->v || !a->pre ||
      !a->area || !a->scalars || !a->p[0])
    return JXB_ERR_ARG;
  if (a->model != 0 && a->model != 1) return JXB_ERR_ARG;
  if (a->model == 0 && (!a->s || !a->p[5])) return JXB_ERR_ARG;
  if (!a->targets_are_nodes && !a->targets) return JXB_ERR_ARG;
  if (a->dtype != JXB_F32 && a->dtype != JXB_F64) return JXB_ERR_DTYPE;
  if (!backward) {
    if (!a->lin || !a->cst) return JXB_ERR_ARG;
    if (a->model == 0 && !a->s_new) return JXB_ERR_ARG;
    if (a->store_current && !a->current) return JXB_ERR_ARG;
  } else {
    if ((!a->accumulate && !a->g_post) || !a->g_lin || !a->g_const || !a->g_v || !a->g_pre || !a->inv ||
        !a->pre_nodes)
      return JXB_ERR_ARG;
    if (a->model == 0 && !a->g_s) return JXB_ERR_ARG;
    if (a->need && !a->g_params) return JXB_ERR_ARG;
  }
  return JXB_OK;
}

}  // namespace

extern "C" int jxb_synapse_forward(const JxbSynArgs* a, void* stream) {
  int rc = check(a, false);
  if (rc) return rc;
  return a->dtype == JXB_F32 ? fwd<float>(*a, (cudaStream_t)stream) : fwd<double>(*a, (cudaStream_t)stream);
}

extern "C" int jxb_synapse_backward(const JxbSynArgs* a, void* stream) {
  int rc = check(a, true);
  if (rc) return rc;
  return a->dtype == JXB_F32 ? bwd<float>(*a, (cudaStream_t)stream) : bwd<double>(*a, (cudaStream_t)stream);
}
