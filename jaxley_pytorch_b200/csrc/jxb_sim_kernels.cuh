// Device code of the fused simulation kernels (forward and adjoint), shared by the
// launchers (jxb_sim.cu) and the units that instantiate the kernels
// (jxb_sim_inst.cu, compiled once per element type, kind and CTA size so that the
// instantiations build in parallel).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include "jxb.h"
#include "jxb_node.cuh"
#include "jxb_prog.cuh"

namespace jxb {

extern thread_local char g_err[512];

void set_err(const char* what, cudaError_t e);

constexpr int kMaxWrites = 24;  // undo-log entries of one node's channel updates
constexpr int FLAG_COMP = 1, FLAG_STIM = 2, FLAG_REC = 4;
constexpr int FLAG_CLAMP = 8;   // the node has clamp entries
constexpr int FLAG_VCLAMP = 16; // one of them clamps v (its last slot holds the unclamped v)

constexpr int kManyKids = 1 << 30;  // chain descriptor flag: more than two child chains

template <typename T>
struct SimSmem {
  // per block
  T *al, *au, *dg, *cm;      // n_nodes
  int* soff;                 // n_nodes, relative to the block's first slot
  short *cls, *poff;         // n_nodes (poff relative to the block's first parameter slot)
  unsigned char* flags;      // n_nodes
  int4* cdesc;               // n_chains: {top, bot | many-children flag, two child tops, parent top}
  int* ccp;                  // n_chains + 1 (relative)
  short* cchild;             // n_child
  int* lp;                   // n_levels + 1
  short *par, *kptr, *kids;  // parent, children CSR (block-relative)
  ChanEntry* ents;
  int* cptr;                 // n_classes + 1 (entries of every node class)
  int* cprog;                // n_classes (compile-time program or PROG_GENERIC)
  T* pb;                     // n_pslots (parameter bases)
  int* pc;                   // n_pslots (parameter columns)
  int* gk;                   // n_pslots (gradient rank or -1)
  const int* gbase;          // n_nodes (first gradient slot), global
  T* gacc;                   // rows * max_gslots (adjoint only)
  // per row
  T *st, *D, *S, *pv;        // rows * (n_slots | n_nodes | n_nodes | n_pslots)
  T* V;                      // rows * n_nodes: voltages during the segment
  // adjoint
  T *adj, *X1;               // rows * n_slots, rows * n_nodes
  unsigned long long* mbar;  // completion barrier of the bulk copies of the state row
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Step of the implicit voltage system: dt for backward Euler, dt / 2 for
// Crank-Nicolson (modules/base.py:3327-3330), whose voltage then moves by twice the
// increment (v' = 2 v_half - v, :3362-3365); the channels always step by dt.
template <typename T>
__host__ __device__ __forceinline__ T solve_dt(const JxbSimArgs& a, T dt) {
  return a.scheme == JXB_SCHEME_CN ? dt * T(0.5) : dt;
}

template <typename T>
__host__ __device__ inline size_t sim_smem_layout(const JxbSimArgs& a, bool backward, SimSmem<T>* o,
                                                  char* base) {
  const size_t R = a.max_rows, nn = a.max_nodes, ns = a.max_slots, nc = a.max_chains,
               nk = a.max_child, nl = a.max_levels, np = a.max_pslots, ne = a.n_entries;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t r = off;
    off = align_up(off + bytes, 16);
    return base ? (void*)(base + r) : nullptr;
  };
  SimSmem<T> s;
  // 8-byte types first.
  // + room to place a row at its source's 16-byte phase and round a bulk copy up to
  // whole 16-byte units
  s.st = (T*)take(sizeof(T) * R * ns + 32);
  s.mbar = backward ? (unsigned long long*)take(16) : nullptr;
  s.adj = backward ? (T*)take(sizeof(T) * R * ns) : nullptr;
  s.D = (T*)take(sizeof(T) * R * nn);
  s.S = (T*)take(sizeof(T) * R * nn);
  s.V = (T*)take(sizeof(T) * R * nn);
  s.X1 = backward ? s.V : nullptr;  // the reverse sweep does not use V
  s.pv = (T*)take(sizeof(T) * R * np);
  s.gacc = (backward && !a.gacc) ? (T*)take(sizeof(T) * R * (size_t)a.max_gslots) : nullptr;
  s.al = (T*)take(sizeof(T) * nn);
  s.au = (T*)take(sizeof(T) * nn);
  // The adjoint reads cm from global memory and forms the diagonal constant on the
  // fly (shared memory goes to more CTAs per SM instead).
  s.dg = backward ? nullptr : (T*)take(sizeof(T) * nn);
  s.cm = backward ? nullptr : (T*)take(sizeof(T) * nn);
  s.pb = (T*)take(sizeof(T) * np);
  s.soff = (int*)take(sizeof(int) * nn);
  s.pc = (int*)take(sizeof(int) * np);
  s.gk = (int*)take(sizeof(int) * np);
  s.cdesc = (int4*)take(sizeof(int4) * nc);
  s.ccp = (int*)take(sizeof(int) * (nc + 1));
  s.lp = (int*)take(sizeof(int) * (nl + 1));
  s.ents = (ChanEntry*)take(sizeof(ChanEntry) * ne);
  s.cptr = (int*)take(sizeof(int) * (a.n_classes + 1));
  s.cprog = (int*)take(sizeof(int) * a.n_classes);
  s.cls = (short*)take(sizeof(short) * nn);
  s.poff = (short*)take(sizeof(short) * nn);
  s.cchild = (short*)take(sizeof(short) * (nk + 1));
  s.par = (short*)take(sizeof(short) * nn);
  s.kptr = (short*)take(sizeof(short) * (nn + 1));
  s.kids = (short*)take(sizeof(short) * (nn + 1));
  s.flags = (unsigned char*)take(nn);
  if (o) *o = s;
  return off;
}

// Stages the block's topology, the channel programs, the parameter values of the
// item's rows and the rows' states (and adjoints) in shared memory.
template <typename T>
__device__ __forceinline__ void stage_item(const JxbSimArgs& a, const JxbBlock& blk, int row0, int rows,
                                           const SimSmem<T>& sm, T dt, const T* state_src, const T* adj_src,
                                           int gslots = 0) {
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nn = blk.n_nodes, ns = blk.n_slots, node0 = blk.node0;
  const T* gl = (const T*)a.a_low;
  const T* gu = (const T*)a.a_up;
  const T* gs = (const T*)a.gsum;
  const T* cmv = (const T*)a.cm;
  dt = solve_dt<T>(a, dt);  // the voltage system's step (half of it for Crank-Nicolson)
  for (int j = tid; j < nn; j += NT) {
    const int i = node0 + j;
    const int cls = a.node_class[i];
    const bool comp = a.cls_comp[cls] != 0;
    sm.al[j] = -(dt * gl[i]);
    sm.au[j] = -(dt * gu[i]);
    if (sm.dg) sm.dg[j] = (comp ? T(1) : T(0)) + dt * gs[i];
    if (sm.cm) sm.cm[j] = cmv[i];
    sm.soff[j] = a.soff[i] - blk.slot0;
    sm.cls[j] = (short)cls;
    sm.poff[j] = (short)(a.poff[i] - blk.pslot0);
    unsigned char f = comp ? FLAG_COMP : 0;
    if (a.stim_ptr[i + 1] > a.stim_ptr[i]) f |= FLAG_STIM;
    if (a.n_rec > 0 && a.rec_ptr[i + 1] > a.rec_ptr[i]) f |= FLAG_REC;
    if (a.clamp_ptr && a.clamp_ptr[i + 1] > a.clamp_ptr[i]) {
      f |= FLAG_CLAMP;
      for (int q = a.clamp_ptr[i]; q < a.clamp_ptr[i + 1]; ++q)
        if (a.clamp_slot[q] == 0) f |= FLAG_VCLAMP;
    }
    sm.flags[j] = f;
    const int pa = a.parent[i];
    sm.par[j] = (short)(pa >= 0 ? pa - node0 : -1);
    sm.kptr[j] = (short)(a.kid_ptr[i] - a.kid_ptr[node0]);
  }
  if (tid == 0) sm.kptr[nn] = (short)(a.kid_ptr[node0 + nn] - a.kid_ptr[node0]);
  {
    const int kb = a.kid_ptr[node0], ke = a.kid_ptr[node0 + nn];
    for (int q = tid; q < ke - kb; q += NT) sm.kids[q] = (short)(a.kid[kb + q] - node0);
  }
  const int nc = blk.n_chains, c0 = blk.chain0;
  const int k0 = a.chain_cptr[c0];
  for (int c = tid; c < nc; c += NT) {
    const int top = a.chain_top[c0 + c] - node0;
    const int len = a.chain_len[c0 + c];
    const int pt = a.chain_ptop[c0 + c];
    const int kb = a.chain_cptr[c0 + c], ke = a.chain_cptr[c0 + c + 1];
    sm.ccp[c] = kb - k0;
    // One 16-byte record per chain: what a solve level reads before its arithmetic.
    unsigned kids = 0xFFFFFFFFu;
    if (ke - kb >= 1) kids = (kids & 0xFFFF0000u) | (unsigned)(a.chain_child[kb] - node0);
    if (ke - kb >= 2) kids = (kids & 0x0000FFFFu) | ((unsigned)(a.chain_child[kb + 1] - node0) << 16);
    sm.cdesc[c] = make_int4(top, (top + len - 1) | (ke - kb > 2 ? kManyKids : 0), (int)kids,
                            pt >= 0 ? pt - node0 : -1);
  }
  if (tid == 0) sm.ccp[nc] = a.chain_cptr[c0 + nc] - k0;
  const int nk = a.chain_cptr[c0 + nc] - k0;
  for (int q = tid; q < nk; q += NT) sm.cchild[q] = (short)(a.chain_child[k0 + q] - node0);
  for (int q = tid; q <= blk.n_levels; q += NT) sm.lp[q] = a.level_ptr[blk.level0 + q];
  const short* src = (const short*)a.entries;
  short* dst = (short*)sm.ents;
  const int nshort = a.n_entries * (int)(sizeof(ChanEntry) / sizeof(short));
  for (int q = tid; q < nshort; q += NT) dst[q] = src[q];
  for (int q = tid; q <= a.n_classes; q += NT) sm.cptr[q] = a.cls_ptr[q];
  for (int q = tid; q < a.n_classes; q += NT) sm.cprog[q] = a.cls_prog ? a.cls_prog[q] : 0;
  const int np = blk.n_pslots;
  const T* pbase = (const T*)a.pbase;
  const T* pscale = (const T*)a.pscale;
  for (int q = tid; q < np; q += NT) {
    sm.pb[q] = pbase[blk.pslot0 + q];
    sm.pc[q] = a.pcol[blk.pslot0 + q];
    sm.gk[q] = a.gk[blk.pslot0 + q];
  }
  for (int w = tid; w < rows * np; w += NT) {
    const int r = w / np, q = w % np;
    const int g = blk.pslot0 + q;
    sm.pv[(size_t)r * np + q] = pbase[g] * pscale[(size_t)(row0 + r) * a.n_cols + a.pcol[g]];
  }
  for (int r = 0; r < rows; ++r) {
    const T* g = state_src + (size_t)(row0 + r) * a.n_slots + blk.slot0;
    T* s = sm.st + (size_t)r * ns;
    for (int q = tid; q < ns; q += NT) s[q] = g[q];
    if (adj_src) {
      const T* ga = adj_src + (size_t)(row0 + r) * a.n_slots + blk.slot0;
      T* sa = sm.adj + (size_t)r * ns;
      for (int q = tid; q < ns; q += NT) sa[q] = ga[q];
    }
  }
  if (sm.gacc) {
    for (int q = tid; q < rows * gslots; q += NT) sm.gacc[q] = T(0);
  }
}

// Voltages of the staged states (after a barrier that follows `stage_item`).
template <typename T>
__device__ __forceinline__ void init_voltages(const JxbBlock& blk, const SimSmem<T>& sm, int rows) {
  const int nn = blk.n_nodes, ns = blk.n_slots;
  for (int w = threadIdx.x; w < nn * rows; w += blockDim.x) {
    const int r = w / nn, j = w - r * nn;
    sm.V[(size_t)r * nn + j] = sm.st[(size_t)r * ns + sm.soff[j]];
  }
}

// Chain recurrences with the coefficients of up to kSeg consecutive nodes loaded
// into registers before the dependent arithmetic (a chain is processed in segments
// of kSeg nodes): the recurrence then waits on arithmetic only, not on a shared
// memory load after every step. The operations and their order are those of the
// node-by-node form.
constexpr int kSeg = 4;

// Elimination of chain c, bottom to top, after its child chains: D receives the
// reciprocal of every pivot, S the eliminated right-hand side.
template <typename T>
__device__ __forceinline__ void chain_eliminate(const SimSmem<T>& sm, int c, T* __restrict__ Dr,
                                                T* __restrict__ Sr, const T* __restrict__ al,
                                                const T* __restrict__ au) {
  const int4 dsc = sm.cdesc[c];
  const int top = dsc.x;
  const int bot = dsc.y & ~kManyKids;
  // The first kSeg nodes above the bottom are loaded together with the bottom and the
  // child chains (indices clamped to the chain: a shorter chain runs its unused
  // lanes on copies of its top node and never stores them).
  const int n0 = min(kSeg, bot - top);
  T dd[kSeg], ss[kSeg], lo[kSeg], up[kSeg];
#pragma unroll
  for (int q = 0; q < kSeg; ++q) {
    const int i = max(bot - 1 - q, top), i1 = min(i + 1, bot);
    dd[q] = Dr[i];
    ss[q] = Sr[i];
    lo[q] = al[i1];
    up[q] = au[i1];
  }
  T d = Dr[bot], s = Sr[bot];
  if (!(dsc.y & kManyKids)) {
    // up to two child chains: their values are loaded together
    const int k0 = dsc.z & 0xFFFF, k1 = (unsigned)dsc.z >> 16;
    T u0 = T(0), q0 = T(0), l0 = T(0), s0 = T(0), u1 = T(0), q1 = T(0), l1 = T(0), s1 = T(0);
    if (k0 != 0xFFFF) { u0 = au[k0]; q0 = Dr[k0]; l0 = al[k0]; s0 = Sr[k0]; }
    if (k1 != 0xFFFF) { u1 = au[k1]; q1 = Dr[k1]; l1 = al[k1]; s1 = Sr[k1]; }
    if (k0 != 0xFFFF) {
      const T f = u0 * q0;
      d -= l0 * f;
      s -= s0 * f;
    }
    if (k1 != 0xFFFF) {
      const T f = u1 * q1;
      d -= l1 * f;
      s -= s1 * f;
    }
  } else {
    for (int k = sm.ccp[c]; k < sm.ccp[c + 1]; ++k) {
      const int ct = sm.cchild[k];
      const T f = au[ct] * Dr[ct];
      d -= al[ct] * f;
      s -= Sr[ct] * f;
    }
  }
  T id = rcp(d);
  Dr[bot] = id;
  Sr[bot] = s;
#pragma unroll
  for (int q = 0; q < kSeg; ++q) {
    const T f = up[q] * id;
    d = dd[q] - lo[q] * f;
    s = ss[q] - s * f;
    id = rcp(d);
    dd[q] = id;
    ss[q] = s;
  }
#pragma unroll
  for (int q = 0; q < kSeg; ++q)
    if (q < n0) {
      Dr[bot - 1 - q] = dd[q];
      Sr[bot - 1 - q] = ss[q];
    }
  // Chains longer than 1 + kSeg continue segment by segment from the recurrence's
  // state after the first kSeg nodes (all of them real then).
  for (int hi = bot - 1 - kSeg; hi >= top; hi -= kSeg) {
    const int n = min(kSeg, hi - top + 1);
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) {
        dd[q] = Dr[hi - q];
        ss[q] = Sr[hi - q];
        lo[q] = al[hi - q + 1];
        up[q] = au[hi - q + 1];
      }
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) {
        const T f = up[q] * id;
        d = dd[q] - lo[q] * f;
        s = ss[q] - s * f;
        id = rcp(d);
        dd[q] = id;
        ss[q] = s;
      }
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) {
        Dr[hi - q] = dd[q];
        Sr[hi - q] = ss[q];
      }
  }
}

// Back-substitution of chain c, top to bottom, from its parent's solution; adds the
// solution to `Vr` when given.
template <typename T>
__device__ __forceinline__ void chain_backsub(const SimSmem<T>& sm, int c, const T* __restrict__ Dr,
                                              T* __restrict__ Sr, const T* __restrict__ al,
                                              T* __restrict__ Vr, T vscale = T(1)) {
  const int4 dsc = sm.cdesc[c];
  const int top = dsc.x;
  const int bot = dsc.y & ~kManyKids;
  const int pt = dsc.w;
  // The first kSeg + 1 nodes in one pass, loads first (indices clamped to the chain,
  // unused lanes never stored), then the rest of a longer chain by segments.
  constexpr int kB = kSeg + 1;
  const int n0 = min(kB, bot - top + 1);
  T db[kB], sb[kB], lb[kB];
#pragma unroll
  for (int q = 0; q < kB; ++q) {
    const int i = min(top + q, bot);
    db[q] = Dr[i];
    sb[q] = Sr[i];
    lb[q] = al[i];
  }
  T xp = pt >= 0 ? Sr[pt] : T(0);
#pragma unroll
  for (int q = 0; q < kB; ++q) {
    const T x = (sb[q] - lb[q] * xp) * db[q];
    sb[q] = x;
    xp = x;
  }
#pragma unroll
  for (int q = 0; q < kB; ++q)
    if (q < n0) {
      Sr[top + q] = sb[q];
      if (Vr) Vr[top + q] += vscale * sb[q];
    }
  for (int l0 = top + kB; l0 <= bot; l0 += kSeg) {
    const int n = min(kSeg, bot - l0 + 1);
    T dd[kSeg], ss[kSeg], ll[kSeg];
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) {
        dd[q] = Dr[l0 + q];
        ss[q] = Sr[l0 + q];
        ll[q] = al[l0 + q];
      }
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) {
        const T x = (ss[q] - ll[q] * xp) * dd[q];
        ss[q] = x;
        xp = x;
      }
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) {
        Sr[l0 + q] = ss[q];
        if (Vr) Vr[l0 + q] += vscale * ss[q];
      }
  }
}

// Chain elimination (leaves first) and back-substitution of every tree of the block
// for all rows. `al`/`au` are A[i, parent] / A[parent, i]. On return `S` holds the
// solution (and `V`, when given, has it added).
template <typename T>
__device__ __forceinline__ void block_solve(const JxbBlock& blk, const SimSmem<T>& sm, int rows,
                                            const T* al, const T* au, T* V = nullptr, T vscale = T(1)) {
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nn = blk.n_nodes;
  const int nlev = blk.n_levels;
  // Elimination, leaf chains first (solver_voltage.py:93-98).
  // (the level table is static: the next level's bounds are read before the barrier)
  int la = sm.lp[0], lb = sm.lp[1];
  for (int h = 0; h < nlev; ++h) {
    const int lc = h + 2 <= nlev ? sm.lp[h + 2] : lb;
    const int c0 = la, nch = lb - la;
    la = lb;
    lb = lc;
    for (int w = tid; w < nch * rows; w += NT) {
      const int r = rows == 1 ? 0 : w / nch;  // no division for one row
      chain_eliminate<T>(sm, c0 + (w - r * nch), sm.D + (size_t)r * nn, sm.S + (size_t)r * nn, al, au);
    }
    __syncthreads();
  }
  // Back-substitution, root chains first (solver_voltage.py:100-106).
  int hb = sm.lp[nlev - 1], he = sm.lp[nlev];
  for (int h = nlev - 1; h >= 0; --h) {
    const int hz = h > 0 ? sm.lp[h - 1] : hb;
    const int c0 = hb, nch = he - hb;
    he = hb;
    hb = hz;
    for (int w = tid; w < nch * rows; w += NT) {
      const int r = rows == 1 ? 0 : w / nch;
      chain_backsub<T>(sm, c0 + (w - r * nch), sm.D + (size_t)r * nn, sm.S + (size_t)r * nn, al,
                       V ? V + (size_t)r * nn : nullptr, vscale);
    }
    __syncthreads();
  }
}

// Channel step of one node and row. mode 0: updates + currents; 1: currents only;
// 2: steady state only. Returns the summed slope and g*E terms in uA/cm^2
// (modules/base.py:3500-3502: mA/cm^2 * 1000).
template <typename T>
__device__ __forceinline__ void node_channels(const SimSmem<T>& sm, int j, T* x, const T* pv, T dt,
                                              int mode, T& lin, T& cst) {
  const int cls = sm.cls[j];
  const int e0 = sm.cptr[cls], e1 = sm.cptr[cls + 1];
  const T* pn = pv + sm.poff[j];
  const T v = x[0];
  lin = cst = T(0);
  if (mode == 0) {
    const int prog = sm.cprog[cls];
    if (prog == PROG_L5PC_DEND) {
      ProgL5pcDend<T>::forward(x, pn, dt, lin, cst);
      return;
    }
    if (prog == PROG_HH) {
      ProgHH<T>::forward(x, pn, dt, lin, cst);
      return;
    }
    if (prog == PROG_L5PC_SOMA) {
      ProgL5pcSoma<T>::forward(x, pn, dt, lin, cst);
      return;
    }
  }
  if (mode == 2) {
    for (int q = e0; q < e1; ++q) channel_steady<T>(sm.ents[q], x, Prm<T>{pn + sm.ents[q].p[0]}, v);
    return;
  }
  if (mode == 0) {
    for (int q = e0; q < e1; ++q) {
      const ChanEntry& e = sm.ents[q];
      channel_update<T>(e, x, Prm<T>{pn + e.p[0]}, v, dt);
    }
  }
  for (int q = e0; q < e1; ++q) {
    const int c = sm.ents[q].cur;
    if (c >= 0) x[c] = T(0);
  }
  T slope = T(0), gge = T(0);
  for (int q = e0; q < e1; ++q) {
    const ChanEntry& e = sm.ents[q];
    channel_current<T>(e, x, Prm<T>{pn + e.p[0]}, v, slope, gge);
  }
  lin = slope * T(1000.0);
  cst = gge * T(1000.0);
}

template <typename T>
__device__ __forceinline__ T stim_current(const JxbSimArgs& a, int i, int b, int t) {
  T acc = T(0);
  if (t >= a.stim_steps) return acc;
  const T* st = (const T*)a.stim + (size_t)t * a.stim_rows * a.n_stim +
                (size_t)(a.stim_rows == 1 ? 0 : b) * a.n_stim;
  const T area = ((const T*)a.area)[i];
  for (int q = a.stim_ptr[i]; q < a.stim_ptr[i + 1]; ++q) acc += fdiv(st[a.stim_idx[q]], area) * T(100000);
  return acc;
}

// Clamp value of entry q for batch row b after step t.
template <typename T>
__device__ __forceinline__ T clamp_value(const JxbSimArgs& a, int q, int b, int t) {
  const T* c = (const T*)a.clamp + ((size_t)t * a.clamp_rows + (a.clamp_rows == 1 ? 0 : b)) * a.n_clamp;
  return c[a.clamp_col[q]];
}

// Clamps of the non-voltage states of node i after the step's channel update
// (modules/base.py:3305-3308): the currents of the step were taken before.
template <typename T>
__device__ __forceinline__ void clamp_states(const JxbSimArgs& a, int i, T* x, int b, int t) {
  for (int q = a.clamp_ptr[i]; q < a.clamp_ptr[i + 1]; ++q) {
    const int sl = a.clamp_slot[q];
    if (sl > 0) x[sl] = clamp_value<T>(a, q, b, t);
  }
}

// Voltage clamps of a block after the solve of step t (modules/base.py:3396-3398):
// a clamped node keeps the solve output in its last slot and takes the clamp value.
template <typename T>
__device__ __forceinline__ void clamp_voltages(const JxbSimArgs& a, const JxbBlock& blk, const SimSmem<T>& sm,
                                               int row0, int rows, int t) {
  const int nn = blk.n_nodes, ns = blk.n_slots;
  for (int w = threadIdx.x; w < nn * rows; w += blockDim.x) {
    const int r = w / nn, j = w - r * nn;
    if (!(sm.flags[j] & FLAG_VCLAMP)) continue;
    const int i = blk.node0 + j;
    const int last = (j + 1 < nn ? sm.soff[j + 1] : ns) - 1;
    T& v = sm.V[(size_t)r * nn + j];
    sm.st[(size_t)r * ns + last] = v;
    for (int q = a.clamp_ptr[i]; q < a.clamp_ptr[i + 1]; ++q)
      if (a.clamp_slot[q] == 0) v = clamp_value<T>(a, q, row0 + r, t);
  }
}

// Slot holding the value after the solve of node j: the last slot of a
// voltage-clamped node, else v.
template <typename T>
__device__ __forceinline__ int solve_slot(const SimSmem<T>& sm, int j, int nn, int ns) {
  return (sm.flags[j] & FLAG_VCLAMP) ? (j + 1 < nn ? sm.soff[j + 1] : ns) - sm.soff[j] - 1 : 0;
}

// Recordings of node i at time index t (integrate.py:53-84).
template <typename T>
__device__ __forceinline__ void record_node(const JxbSimArgs& a, int i, const T* x, int b, int t) {
  T* out = (T*)a.rec_out;
  for (int q = a.rec_ptr[i]; q < a.rec_ptr[i + 1]; ++q) {
    const int sl = a.rec_slot[q];
    out[((size_t)t * a.batch + b) * a.n_rec + a.rec_col[q]] = sl >= 0 ? x[sl] : T(0);
  }
}


// The (row, node) pairs one thread visits in a per-node phase. With a node schedule
// for this launch's warp count, warp w visits its listed nodes (each chunk of 32
// lanes holds nodes of one class; the chunks are balanced over the warps by cost),
// every row of a node in turn; otherwise the pairs are strided over the threads.
struct NodeWalk {
  const short* sc;  // schedule of this thread (stride 32), or null
  int n;            // visits
  int rows, nn, w0, stride;

  __device__ __forceinline__ NodeWalk(const JxbSimArgs& a, const JxbBlock& blk, int rows_, int item_block) {
    const int tid = threadIdx.x, NT = blockDim.x;
    rows = rows_;
    nn = blk.n_nodes;
    if (a.sched && a.sched_warps * 32 == NT) {
      const int s0 = a.sched_ptr[item_block], s1 = a.sched_ptr[item_block + 1];
      const int per_warp = (s1 - s0) / a.sched_warps;  // iterations x 32
      sc = a.sched + s0 + (tid >> 5) * per_warp + (tid & 31);
      n = per_warp / 32 * rows;
      w0 = stride = 0;
    } else {
      sc = nullptr;
      w0 = tid;
      stride = NT;
      n = tid < nn * rows ? (nn * rows - tid + NT - 1) / NT : 0;
    }
  }
  // (r, j) of visit q; false for an idle lane.
  __device__ __forceinline__ bool get(int q, int& r, int& j) const {
    if (sc) {
      const int k = rows == 1 ? q : q / rows;
      r = q - k * rows;
      j = __ldg(sc + k * 32);
      return j >= 0;
    }
    const int w = w0 + q * stride;
    r = rows == 1 ? 0 : w / nn;
    j = w - r * nn;
    return true;
  }
};

// Runs `n_steps` forward steps of one item from the staged state. Used by the
// forward kernel (ckpt/rec outputs) and by the adjoint (trajectory store).
// On return sm.st holds the state after the last step; `X1` (if not null) receives
// the final voltages.
template <typename T>
__device__ __forceinline__ void run_steps(const JxbSimArgs& a, const JxbBlock& blk, int item_block, int row0,
                                          int rows, const SimSmem<T>& sm, T dt, int t0, int nsteps, int mode,
                                          bool record, bool ckpt, T* traj, T* X1, T* piv = nullptr,
                                          bool traj_final = false) {
  const int nn = blk.n_nodes, ns = blk.n_slots, np = blk.n_pslots;
  const NodeWalk walk(a, blk, rows, item_block);  // the same visits every step
  const T dts = solve_dt<T>(a, dt);               // step of the voltage system
  const T vscale = a.scheme == JXB_SCHEME_CN ? T(2) : T(1);  // v' = v + vscale * increment
  // Whether any node of the block has a voltage clamp (uniform over the CTA).
  int mine = 0;
  if (a.clamp_ptr)
    for (int j = threadIdx.x; j < nn; j += blockDim.x) mine |= sm.flags[j] & FLAG_VCLAMP;
  const bool vclamps = __syncthreads_or(mine) != 0;
  for (int step = 0; step <= nsteps; ++step) {
    const int t = t0 + step;
    for (int q = 0; q < walk.n; ++q) {
      int r, j;
      if (!walk.get(q, r, j)) continue;
      const int i = blk.node0 + j;
      const int b = row0 + r;
      T* x = sm.st + (size_t)r * ns + sm.soff[j];
      const int nslot = (j + 1 < nn ? sm.soff[j + 1] : ns) - sm.soff[j];
      const unsigned char f = sm.flags[j];
      const T* Vr = sm.V + (size_t)r * nn;
      if (step > 0) x[0] = Vr[j];
      if (piv && step > 0)  // reciprocal pivots of the previous step's elimination
        piv[((size_t)(step - 1) * a.batch + b) * a.n_nodes + i] = sm.D[(size_t)r * nn + j];
      if (record && step > 0 && (f & FLAG_REC)) record_node<T>(a, i, x, b, t);
      if (step == nsteps) {
        if (traj_final) {  // the state after the last step closes the trajectory
          T* g = traj + ((size_t)nsteps * a.batch + b) * a.n_slots + blk.slot0 + sm.soff[j];
          for (int q = 0; q < nslot; ++q) g[q] = x[q];
        }
        if (mode != 0) {
          T lin, cst;
          if (mode == 2) node_channels<T>(sm, j, x, sm.pv + (size_t)r * np, dt, 2, lin, cst);
          node_channels<T>(sm, j, x, sm.pv + (size_t)r * np, dt, 1, lin, cst);
          if (record && (f & FLAG_REC)) record_node<T>(a, i, x, b, t);
        }
        if (X1) X1[(size_t)r * nn + j] = (f & FLAG_VCLAMP) ? x[nslot - 1] : x[0];
        continue;
      }
      if (traj) {
        T* g = traj + ((size_t)step * a.batch + b) * a.n_slots + blk.slot0 + sm.soff[j];
        for (int q = 0; q < nslot; ++q) g[q] = x[q];
      }
      if (ckpt && ((t - a.ckpt_base) % a.ckpt_every) == 0) {
        const size_t m = (size_t)((t - a.ckpt_base) / a.ckpt_every);
        T* g = (T*)a.ckpt + (m * a.batch + b) * a.n_slots + blk.slot0 + sm.soff[j];
        for (int q = 0; q < nslot; ++q) g[q] = x[q];
      }
      const T v = x[0];
      T lin, cst;
      node_channels<T>(sm, j, x, sm.pv + (size_t)r * np, dt, 0, lin, cst);
      if (f & FLAG_CLAMP) clamp_states<T>(a, i, x, b, t);
      if (f & FLAG_STIM) cst += stim_current<T>(a, i, b, t);
      if (a.syn_lin) {
        if (a.syn_ptr) {  // per-target synapse outputs (modules/network.py:402-407)
          for (int q = a.syn_ptr[i]; q < a.syn_ptr[i + 1]; ++q) {
            const size_t o = (size_t)a.syn_off[q] + (size_t)b * a.syn_rs[q];
            lin += ((const T*)a.syn_lin)[o];
            cst -= ((const T*)a.syn_const)[o];
          }
        } else {
          lin += ((const T*)a.syn_lin)[(size_t)b * a.n_nodes + i];
          cst += ((const T*)a.syn_const)[(size_t)b * a.n_nodes + i];
        }
      }
      const T cmv = sm.cm[j];
      // Delta form of the implicit step: A (v' - v) = rhs - A v, with
      // (A v)_j = d_j v_j + sum over neighbours of the off-diagonals times their v,
      // written with voltage differences (exact algebra, small increments).
      const T lin_t = dts * fdiv(lin, cmv);
      T axv = T(0);
      const int pj = sm.par[j];
      if (pj >= 0) axv += sm.al[j] * (Vr[pj] - v);
      for (int k = sm.kptr[j]; k < sm.kptr[j + 1]; ++k) {
        const int c = sm.kids[k];
        axv += sm.au[c] * (Vr[c] - v);
      }
      const T dgj = sm.dg ? sm.dg[j] : ((f & FLAG_COMP) ? T(1) : T(0)) + dts * ((const T*)a.gsum)[i];
      sm.D[(size_t)r * nn + j] = dgj + lin_t;
      sm.S[(size_t)r * nn + j] = ((f & FLAG_COMP) ? dts * fdiv(cst, cmv) - lin_t * v : T(0)) - axv;
    }
    if (step == nsteps) break;
    __syncthreads();
    block_solve<T>(blk, sm, rows, sm.al, sm.au, sm.V, vscale);
    if (vclamps) {
      clamp_voltages<T>(a, blk, sm, row0, rows, t);
      __syncthreads();
    }
  }
  __syncthreads();
}

// ORs JXB_NONFINITE into the launch's status flag when any thread of the CTA saw a
// value that is not finite (all threads of the CTA call this).
__device__ __forceinline__ void report_nonfinite(const JxbSimArgs& a, int bad) {
  if (__syncthreads_or(bad) && threadIdx.x == 0 && a.status) atomicOr(a.status, JXB_NONFINITE);
}

// Work areas of the CTA: dynamic shared memory, or (GM) the item's range of the
// caller's global scratch for blocks too large for shared memory.
template <bool GM>
__device__ __forceinline__ char* work_base(const JxbSimArgs& a, char* smem_raw) {
  if constexpr (GM) return (char*)a.gscratch + (size_t)blockIdx.x * (size_t)a.gscratch_stride;
  return smem_raw;
}

// Forward launch of one work item: `a` describes the problem (a request), `L` the
// launch (work-area sizing, global scratch).
template <typename T, bool GM>
__device__ __forceinline__ void sim_forward_body(const JxbSimArgs& a, const JxbSimArgs& L, int item_idx,
                                                 char* smem_raw) {
  SimSmem<T> sm;
  sim_smem_layout<T>(L, false, &sm, work_base<GM>(L, smem_raw));
  const JxbItem item = a.items[item_idx];
  const JxbBlock blk = a.blocks[item.block];
  const int rows = item.n_rows, row0 = item.row0;
  const T dt = T(a.dt);
  stage_item<T>(a, blk, row0, rows, sm, dt, (const T*)a.state, nullptr);
  __syncthreads();
  init_voltages<T>(blk, sm, rows);
  __syncthreads();
  const int nsteps = a.mode == 0 ? a.n_steps : 0;
  // With `traj`, the launch also stores the state before every step, the state after
  // the last one and the reciprocal pivots of every step (`traj_piv`), for an
  // adjoint that then skips its recompute (`traj_stored`).
  run_steps<T>(a, blk, item.block, row0, rows, sm, dt, a.t0, nsteps, a.mode, a.n_rec > 0, a.ckpt != nullptr,
               (T*)a.traj, nullptr, (T*)a.traj_piv, a.traj != nullptr && nsteps > 0);
  // Write the resident states back (and flag values that are not finite).
  const int ns = blk.n_slots;
  int bad = 0;
  for (int r = 0; r < rows; ++r) {
    T* g = (T*)a.state + (size_t)(row0 + r) * a.n_slots + blk.slot0;
    const T* s = sm.st + (size_t)r * ns;
    for (int q = threadIdx.x; q < ns; q += blockDim.x) {
      const T val = s[q];
      g[q] = val;
      bad |= !is_finite(val);
    }
  }
  report_nonfinite(a, bad);
}

// Adjoint of one node and row for one step: replays the channel updates from the
// pre-step state `x`, logging every overwritten slot with its partial derivatives
// (one evaluation of the rate functions, in dual arithmetic), then applies the VJPs
// of the currents at the updated state and of the updates in reverse order,
// restoring `x` from the log.
template <typename T>
__device__ __forceinline__ void node_adjoint(const SimSmem<T>& sm, int j, T* x, T* lam,
                                             const T* pv, T* gacc, T dt, T lr, T x1,
                                             T& lv) {
  const int cls = sm.cls[j];
  const int e0 = sm.cptr[cls], e1 = sm.cptr[cls + 1];
  const T* pn = pv + sm.poff[j];
  const T* pb = sm.pb + sm.poff[j];
  const int* pk = sm.gk + sm.poff[j];
  T* ga = gacc + sm.gbase[j];
  const int prog = sm.cprog[cls];
  if (prog != PROG_GENERIC) {
    AdjCtx<T> c{lam, pb, pk, ga, lr, x1, lv};
    if (prog == PROG_L5PC_DEND)
      ProgL5pcDend<T>::adjoint(x, pn, dt, c);
    else if (prog == PROG_L5PC_SOMA)
      ProgL5pcSoma<T>::adjoint(x, pn, dt, c);
    else
      ProgHH<T>::adjoint(x, pn, dt, c);
    lv = c.lv;
    return;
  }
  const T v = x[0];
  UndoLog<T, kMaxWrites> L;
  for (int q = e0; q < e1; ++q) {
    const ChanEntry& e = sm.ents[q];
    channel_update_logged<T, kMaxWrites>(e, x, Prm<T>{pn + e.p[0]}, v, dt, L);
  }
  for (int q = e1 - 1; q >= e0; --q) {
    const ChanEntry& e = sm.ents[q];
    PGradSink<T> G{pb + e.p[0], pk + e.p[0], ga};
    channel_current_vjp<T>(e, x, lam, Prm<T>{pn + e.p[0]}, G, v, lr, x1, lv);
  }
  // The step overwrote the current slots, so the adjoint of their previous values
  // starts from zero.
  for (int q = e0; q < e1; ++q) {
    const int c = sm.ents[q].cur;
    if (c >= 0) lam[c] = T(0);
  }
  for (int q = e1 - 1; q >= e0; --q) {
    const ChanEntry& e = sm.ents[q];
    PGradSink<T> G{pb + e.p[0], pk + e.p[0], ga};
    channel_update_vjp_logged<T, kMaxWrites>(e, x, lam, Prm<T>{pn + e.p[0]}, G, v, dt, lv, L);
  }
}

// Adjoint of the initial channel currents of node j: the current slots of the
// initial state are the channel currents at that state (`_append_currents_with_plan`,
// modules/base.py:2375-2383, inside the reference's differentiated integrate), so
// their adjoint (from the first step's reads, e.g. the calcium pump's, and from the
// recordings at t = 0) flows to the channel parameters. The slots' adjoint is then
// consumed: they are outputs of this computation, not inputs.
template <typename T>
__device__ __forceinline__ void node_initial_current_adjoint(const SimSmem<T>& sm, int j, const T* x, T* lam,
                                                             const T* pv, T* gacc) {
  const int cls = sm.cls[j];
  const int e0 = sm.cptr[cls], e1 = sm.cptr[cls + 1];
  const T* pn = pv + sm.poff[j];
  const T* pb = sm.pb + sm.poff[j];
  const int* pk = sm.gk + sm.poff[j];
  T* ga = gacc + sm.gbase[j];
  const T v = x[0];
  T lv = T(0);
  for (int q = e0; q < e1; ++q) {
    const ChanEntry& e = sm.ents[q];
    if (e.cur < 0) continue;
    PGradSink<T> G{pb + e.p[0], pk + e.p[0], ga};
    channel_current_vjp<T>(e, x, lam, Prm<T>{pn + e.p[0]}, G, v, T(0), v, lv);
  }
  lam[0] += lv;
  for (int q = e0; q < e1; ++q) {
    const int c = sm.ents[q].cur;
    if (c >= 0) lam[c] = T(0);
  }
}

// Elimination of chain c for the transposed system with the stored reciprocal
// pivots: only the right-hand side is eliminated.
template <typename T>
__device__ __forceinline__ void chain_eliminate_rhs(const SimSmem<T>& sm, int c, const T* __restrict__ Dr,
                                                    T* __restrict__ Sr, const T* __restrict__ au) {
  const int4 dsc = sm.cdesc[c];
  const int top = dsc.x;
  const int bot = dsc.y & ~kManyKids;
  // First segment loaded with the bottom and the child chains (as chain_eliminate).
  const int n0 = min(kSeg, bot - top);
  T ss[kSeg], up[kSeg], dn[kSeg];
#pragma unroll
  for (int q = 0; q < kSeg; ++q) {
    const int i = max(bot - 1 - q, top), i1 = min(i + 1, bot);
    ss[q] = Sr[i];
    up[q] = au[i1];
    dn[q] = Dr[i1];
  }
  T s = Sr[bot];
  if (!(dsc.y & kManyKids)) {
    const int k0 = dsc.z & 0xFFFF, k1 = (unsigned)dsc.z >> 16;
    T s0 = T(0), u0 = T(0), q0 = T(0), s1 = T(0), u1 = T(0), q1 = T(0);
    if (k0 != 0xFFFF) { s0 = Sr[k0]; u0 = au[k0]; q0 = Dr[k0]; }
    if (k1 != 0xFFFF) { s1 = Sr[k1]; u1 = au[k1]; q1 = Dr[k1]; }
    if (k0 != 0xFFFF) s -= s0 * (u0 * q0);
    if (k1 != 0xFFFF) s -= s1 * (u1 * q1);
  } else {
    for (int k = sm.ccp[c]; k < sm.ccp[c + 1]; ++k) {
      const int ct = sm.cchild[k];
      s -= Sr[ct] * (au[ct] * Dr[ct]);
    }
  }
  Sr[bot] = s;
#pragma unroll
  for (int q = 0; q < kSeg; ++q) {
    s = ss[q] - s * (up[q] * dn[q]);
    ss[q] = s;
  }
#pragma unroll
  for (int q = 0; q < kSeg; ++q)
    if (q < n0) Sr[bot - 1 - q] = ss[q];
  for (int hi = bot - 1 - kSeg; hi >= top; hi -= kSeg) {
    const int n = min(kSeg, hi - top + 1);
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) {
        ss[q] = Sr[hi - q];
        up[q] = au[hi - q + 1];
        dn[q] = Dr[hi - q + 1];
      }
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) {
        s = ss[q] - s * (up[q] * dn[q]);
        ss[q] = s;
      }
#pragma unroll
    for (int q = 0; q < kSeg; ++q)
      if (q < n) Sr[hi - q] = ss[q];
  }
}

// Transposed solve with the reciprocal pivots of the forward elimination (the
// pivots of A and A^T coincide): only the right-hand side is eliminated. Levels as in
// `block_solve`.
template <typename T>
__device__ __forceinline__ void block_solve_pivots(const JxbBlock& blk, const SimSmem<T>& sm, int rows,
                                                   const T* al, const T* au) {
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nn = blk.n_nodes;
  const int nlev = blk.n_levels;
  int la = sm.lp[0], lb = sm.lp[1];
  for (int h = 0; h < nlev; ++h) {
    const int lc = h + 2 <= nlev ? sm.lp[h + 2] : lb;
    const int c0 = la, nch = lb - la;
    la = lb;
    lb = lc;
    for (int w = tid; w < nch * rows; w += NT) {
      const int r = rows == 1 ? 0 : w / nch;  // no division for one row
      chain_eliminate_rhs<T>(sm, c0 + (w - r * nch), sm.D + (size_t)r * nn, sm.S + (size_t)r * nn, au);
    }
    __syncthreads();
  }
  int hb = sm.lp[nlev - 1], he = sm.lp[nlev];
  for (int h = nlev - 1; h >= 0; --h) {
    const int hz = h > 0 ? sm.lp[h - 1] : hb;
    const int c0 = hb, nch = he - hb;
    he = hb;
    hb = hz;
    for (int w = tid; w < nch * rows; w += NT) {
      const int r = rows == 1 ? 0 : w / nch;
      chain_backsub<T>(sm, c0 + (w - r * nch), sm.D + (size_t)r * nn, sm.S + (size_t)r * nn, al,
                       (T*)nullptr);
    }
    __syncthreads();
  }
}

// Asynchronous element copies global -> shared (cp.async, 4 or 8 bytes: the rows
// are only element-aligned), committed as one group and awaited with
// cp_async_wait_all before a barrier.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem_dst, const T* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "element copies of 4 or 8 bytes");
  if constexpr (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Bulk copies global -> shared (the copy engine, one instruction for a whole row)
// completing on an mbarrier; no cluster multicast.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(m)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* m, unsigned bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(
                   smem_addr(m)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(m))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* m, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of `m` at most kMaxWaitPolls polls; false when it gave up
// (the launch then reports JXB_TIMEOUT instead of hanging).
constexpr int kMaxWaitPolls = 1 << 20;
__device__ __forceinline__ bool mbar_wait(unsigned long long* m, unsigned parity) {
  for (int i = 0; i < kMaxWaitPolls; ++i)
    if (mbar_try_wait(m, parity)) return true;
  return false;
}

// Orders this thread's earlier ordinary accesses (shared and global) before later
// bulk copies; every thread calls it before the barrier that precedes a copy.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;\n" ::: "memory"); }

// Issues (thread 0) the bulk copy of `cnt` elements at `src` into the row buffer
// `base` (16-byte aligned, 32 bytes longer than the row) so that element 0 lands at
// base + shift, where shift puts the row at its source's 16-byte phase; the copy is
// widened to whole 16-byte units on both ends. Every thread gets the shift.
template <typename T>
__device__ __forceinline__ int bulk_stage_row(T* base, const T* src, int cnt, unsigned long long* m) {
  const int shift = (int)(((uintptr_t)src & 15) / sizeof(T));
  const unsigned bytes = (unsigned)(((size_t)(cnt + shift) * sizeof(T) + 15) & ~(size_t)15);
  if (threadIdx.x == 0) {
    mbar_expect_tx(m, bytes);
    bulk_copy_g2s(base, src - shift, bytes, m);
  }
  return shift;
}

// Stages one contiguous range of `cnt` elements asynchronously: 16-byte copies for
// the part where source and destination share their 16-byte phase, element copies
// for the ends (and for the whole range when the phases differ).
template <typename T>
__device__ __forceinline__ void stage_range_async(T* dst, const T* src, int cnt) {
  constexpr int V = 16 / (int)sizeof(T);
  int head = cnt, nvec = 0;
  if ((((uintptr_t)dst ^ (uintptr_t)src) & 15) == 0) {
    head = min(cnt, (int)(((16 - ((uintptr_t)src & 15)) & 15) / sizeof(T)));
    nvec = (cnt - head) / V;
  }
  for (int q = threadIdx.x; q < head; q += blockDim.x) cp_async_elem(dst + q, src + q);
  for (int q = threadIdx.x; q < nvec; q += blockDim.x) cp_async16(dst + head + q * V, src + head + q * V);
  for (int q = head + nvec * V + threadIdx.x; q < cnt; q += blockDim.x) cp_async_elem(dst + q, src + q);
}

// Stages the item's rows of a (steps, batch, width) array at `step` (the block's
// range starting at `off`, `cnt` wide) into shared memory rows of stride `cnt`.
template <typename T>
__device__ __forceinline__ void stage_rows_async(T* dst, const T* src, int step, int batch, int width, int off,
                                                 int cnt, int row0, int rows) {
  for (int r = 0; r < rows; ++r)
    stage_range_async<T>(dst + (size_t)r * cnt, src + ((size_t)step * batch + row0 + r) * width + off, cnt);
  cp_async_commit();
}

// Adjoint launch of one work item (`a`: the problem, `L`: the launch).
template <typename T, bool GM>
__device__ __forceinline__ void sim_backward_body(const JxbSimArgs& a, const JxbSimArgs& L, int item_idx,
                                                  char* smem_raw) {
  SimSmem<T> sm;
  sim_smem_layout<T>(L, true, &sm, work_base<GM>(L, smem_raw));
  const JxbItem item = a.items[item_idx];
  const JxbBlock blk = a.blocks[item.block];
  sm.gbase = a.gbase + blk.node0;
  if (L.gacc) sm.gacc = (T*)((char*)L.gacc + (size_t)blockIdx.x * (size_t)L.gacc_stride);
  // One-row items stage each step's state row with one bulk copy (rows of a multiple
  // of 16 bytes: the copy, widened to 16-byte units, stays inside the row).
  T* const st_base = sm.st;
  bool bulk = !GM && item.n_rows == 1 && (a.n_slots * (int)sizeof(T)) % 16 == 0 && a.traj != nullptr &&
              ((uintptr_t)a.traj & 15) == 0;
  if (bulk) sm.st = st_base + blk.slot0 % (16 / (int)sizeof(T));
  const int gslots = L.max_gslots;
  const int rows = item.n_rows, row0 = item.row0;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int nn = blk.n_nodes, ns = blk.n_slots, np = blk.n_pslots;
  const T dt = T(a.dt);
  const T dts = solve_dt<T>(a, dt);  // step of the voltage system
  const bool cn = a.scheme == JXB_SCHEME_CN;
  const int K = a.n_steps;
  T* traj = (T*)a.traj;
  stage_item<T>(a, blk, row0, rows, sm, dt, (const T*)a.ckpt, (const T*)a.adj, gslots);
  __syncthreads();
  T* piv = (T*)a.traj_piv;
  if (a.traj_stored) {
    // The forward stored the segment's states (entries 0..K) and pivots: the final
    // voltages are those of entry K.
    for (int w = tid; w < nn * rows; w += nthr) {
      const int r = w / nn, j = w - r * nn;
      sm.X1[(size_t)r * nn + j] = traj[((size_t)K * a.batch + row0 + r) * a.n_slots + blk.slot0 + sm.soff[j] +
                                       solve_slot<T>(sm, j, nn, ns)];
    }
    sm.cm = (T*)a.cm + blk.node0;  // read only
    __syncthreads();
  } else {
    // Recompute the segment from its checkpoint, storing the state before every step.
    init_voltages<T>(blk, sm, rows);
    __syncthreads();
    sm.cm = (T*)a.cm + blk.node0;  // read only
    run_steps<T>(a, blk, item.block, row0, rows, sm, dt, a.t0, K, 0, false, false, traj, sm.X1, piv);
  }

  const T* rec_grad = (const T*)a.rec_grad;
  const int total = nn * rows;
  const NodeWalk walk(a, blk, rows, item.block);  // the same visits every step
  // Shared-memory kernels stage each step's pivots (into D, during the previous
  // step's phase 4, which does not use D) and its states (into st, during phase 1
  // and the transposed solve, which do not use st) asynchronously, so that the
  // per-node phases do not wait on global memory.
  if constexpr (!GM) {
    if (bulk && tid == 0) mbar_init(sm.mbar, 1);
    stage_rows_async<T>(sm.D, piv, K - 1, a.batch, a.n_nodes, blk.node0, nn, row0, rows);
    cp_async_wait_all();
    if (bulk) fence_proxy_async();  // the recompute's trajectory stores before the copies
    __syncthreads();
  }
  unsigned parity = 0;  // phase of the state-row barrier the next wait expects
  int timed_out = 0;
  for (int step = K - 1; step >= 0; --step) {
    const int t = a.t0 + step;
    if constexpr (!GM) {
      if (bulk)
        sm.st = st_base + bulk_stage_row<T>(st_base, traj + ((size_t)step * a.batch + row0) * a.n_slots +
                                                         blk.slot0, ns, sm.mbar);
      else
        stage_rows_async<T>(sm.st, traj, step, a.batch, a.n_slots, blk.slot0, ns, row0, rows);
    }
    // Phase 1: recording gradients at t + 1, the pivots of the step's matrix and the
    // right-hand side of the transposed solve.
    for (int w = tid; w < total; w += nthr) {
      const int r = w / nn, j = w - r * nn;
      const int i = blk.node0 + j;
      const int b = row0 + r;
      T* lam = sm.adj + (size_t)r * ns + sm.soff[j];
      const unsigned char f = sm.flags[j];
      if (rec_grad && (f & FLAG_REC)) {
        for (int q = a.rec_ptr[i]; q < a.rec_ptr[i + 1]; ++q) {
          const int sl = a.rec_slot[q];
          if (sl >= 0) lam[sl] += rec_grad[((size_t)(t + 1) * a.batch + b) * a.n_rec + a.rec_col[q]];
        }
      }
      if constexpr (GM) sm.D[(size_t)r * nn + j] = piv[((size_t)step * a.batch + b) * a.n_nodes + i];
      // a clamped voltage after the step does not depend on the solve
      sm.S[(size_t)r * nn + j] = (f & FLAG_VCLAMP) ? T(0) : (cn ? T(2) * lam[0] : lam[0]);
    }
    __syncthreads();
    // lambda_r = A^{-T} lambda_v'  (solver_voltage.py:168-187), with the pivots of
    // the forward elimination.
    block_solve_pivots<T>(blk, sm, rows, sm.au, sm.al);
    if constexpr (!GM) {
      cp_async_wait_all();  // the step's states (element copies)
      if (bulk) {           // the step's states (bulk copy)
        if (!mbar_wait(sm.mbar, parity)) timed_out = 1;
        parity ^= 1u;
      }
      __syncthreads();
      if (step > 0) stage_rows_async<T>(sm.D, piv, step - 1, a.batch, a.n_nodes, blk.node0, nn, row0, rows);
    }
    // Phase 4: vector-Jacobian products of the step.
    for (int q = 0; q < walk.n; ++q) {
      int r, j;
      if (!walk.get(q, r, j)) continue;
      const int b = row0 + r;
      T* x = sm.st + (size_t)r * ns + sm.soff[j];
      T* lam = sm.adj + (size_t)r * ns + sm.soff[j];
      const int nslot = (j + 1 < nn ? sm.soff[j + 1] : ns) - sm.soff[j];
      if constexpr (GM) {
        const T* g = traj + ((size_t)step * a.batch + b) * a.n_slots + blk.slot0 + sm.soff[j];
        for (int q = 0; q < nslot; ++q) x[q] = g[q];
      }
      (void)nslot;
      const T lr = sm.S[(size_t)r * nn + j];
      // the solve's output: v' (backward Euler) or v_half = (v' + v) / 2 (Crank-Nicolson)
      const T xnew = cn ? T(0.5) * (sm.X1[(size_t)r * nn + j] + x[0]) : sm.X1[(size_t)r * nn + j];
      const bool comp = (sm.flags[j] & FLAG_COMP) != 0;
      // d = dg + dt * lin / cm,  rhs = v + dt * cst / cm (compartments only; the
      // branchpoints have no channels); dt is the system's step.
      const T lrs = fdiv(T(1000.0) * dts * lr, sm.cm[j]);
      T lv = comp ? lr : T(0);
      // Crank-Nicolson's v' = 2 v_half - v: the adjoint of v' also reaches v directly
      if (cn && !(sm.flags[j] & FLAG_VCLAMP)) lv -= lam[0];
      if (a.g_syn_lin && a.syn_ptr) {
        // d loss / d (synaptic slope, offset) of node j: the slope enters the
        // diagonal (and, on compartments, the right-hand side as -lin * v), the
        // offset the right-hand side with a minus sign.
        const int i = blk.node0 + j;
        const T f = fdiv(lr * dts, sm.cm[j]);
        const T gl = comp ? -f * xnew : -f * (xnew - x[0]);
        const T gc = comp ? -f : T(0);
        for (int q = a.syn_ptr[i]; q < a.syn_ptr[i + 1]; ++q) {
          const size_t o = (size_t)a.syn_off[q] + (size_t)b * a.syn_rs[q];
          ((T*)a.g_syn_lin)[o] = gl;
          ((T*)a.g_syn_const)[o] = gc;
        }
      }
      lam[0] = T(0);
      if (sm.flags[j] & FLAG_CLAMP) {  // clamped states after the step are constants
        const int i = blk.node0 + j;
        for (int q = a.clamp_ptr[i]; q < a.clamp_ptr[i + 1]; ++q)
          if (a.clamp_slot[q] > 0) lam[a.clamp_slot[q]] = T(0);
      }
      node_adjoint<T>(sm, j, x, lam, sm.pv + (size_t)r * np,
                      sm.gacc + (size_t)r * gslots, dt, lrs, xnew, lv);
      lam[0] = lv;
      sm.X1[(size_t)r * nn + j] = x[solve_slot<T>(sm, j, nn, ns)];
    }
    if constexpr (!GM) {
      cp_async_wait_all();            // the next step's pivots
      if (bulk) fence_proxy_async();  // this step's accesses to the state row before the next copy
    }
    __syncthreads();
  }
  if (a.t0 == 0) {
    // The segment that starts the run: the recordings of t = 0 and the adjoint of the
    // initial currents (the state in `st` is the initial state now).
    for (int w = tid; w < total; w += nthr) {
      const int r = w / nn, j = w - r * nn;
      const int i = blk.node0 + j;
      const int b = row0 + r;
      T* x = sm.st + (size_t)r * ns + sm.soff[j];
      T* lam = sm.adj + (size_t)r * ns + sm.soff[j];
      if constexpr (GM) {
        const int nslot = (j + 1 < nn ? sm.soff[j + 1] : ns) - sm.soff[j];
        const T* g = traj + ((size_t)b) * a.n_slots + blk.slot0 + sm.soff[j];
        for (int q = 0; q < nslot; ++q) x[q] = g[q];
      }
      if (rec_grad && (sm.flags[j] & FLAG_REC)) {
        for (int q = a.rec_ptr[i]; q < a.rec_ptr[i + 1]; ++q) {
          const int sl = a.rec_slot[q];
          if (sl >= 0) lam[sl] += rec_grad[(size_t)b * a.n_rec + a.rec_col[q]];
        }
      }
      node_initial_current_adjoint<T>(sm, j, x, lam, sm.pv + (size_t)r * np, sm.gacc + (size_t)r * gslots);
    }
    __syncthreads();
  }
  // A bulk copy whose wait gave up may still be in flight: wait for it once more
  // (bounded) before the CTA leaves, and report the timeout.
  if (__syncthreads_or(timed_out)) {
    if (bulk) mbar_wait(sm.mbar, parity ^ 1u);
    if (tid == 0 && a.status) atomicOr(a.status, JXB_TIMEOUT);
  }
  int bad = 0;  // a value that is not finite seen by this thread
  // Fold the nodes' gradient slots into the columns (float64, global), once per
  // launch: a shared per-column buffer would scale with the number of columns,
  // which is large when every cell has its own trainable group.
  for (int w = tid; w < total; w += nthr) {
    const int r = w / nn, j = w - r * nn;
    const int cls = sm.cls[j];
    int npar = 0;
    for (int q = sm.cptr[cls]; q < sm.cptr[cls + 1]; ++q) npar += sm.ents[q].np;
    const int po = sm.poff[j];
    const T* ga = sm.gacc + (size_t)r * gslots + sm.gbase[j];
    double* pg = a.pgrad + (size_t)(row0 + r) * a.n_cols;
    for (int k = 0; k < npar; ++k) {
      const int q = sm.gk[po + k];
      if (q >= 0 && ga[q] != T(0)) {
        bad |= !is_finite(ga[q]);
        atomicAdd(pg + sm.pc[po + k], (double)ga[q]);
      }
    }
  }
  // Adjoint of the segment's initial state.
  for (int r = 0; r < rows; ++r) {
    T* ga = (T*)a.adj + (size_t)(row0 + r) * a.n_slots + blk.slot0;
    const T* sa = sm.adj + (size_t)r * ns;
    for (int q = tid; q < ns; q += nthr) {
      const T val = sa[q];
      ga[q] = val;
      bad |= !is_finite(val);
    }
  }
  report_nonfinite(a, bad);
}

// Arguments of a request in a multi-request launch, copied into shared memory.
template <typename T>
__device__ JxbSimArgs& request_args_slot() {
  __shared__ JxbSimArgs s;
  return s;
}

// A launch runs the items of one problem (`L.items`), or, with `L.multi`, the
// (request, item) pairs `L.multi_items` of several problems whose arguments are in
// `L.multi` (continuous batching of requests); the work-area sizing and global
// scratch are the launch's.
template <typename T, bool MULTI>
__device__ __forceinline__ const JxbSimArgs& item_args(const JxbSimArgs& L, int& item_idx) {
  item_idx = blockIdx.x;
  if constexpr (MULTI) {
    JxbSimArgs& s = request_args_slot<T>();
    const int2 mi = reinterpret_cast<const int2*>(L.multi_items)[blockIdx.x];
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(L.multi + mi.x);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&s);
    for (int q = threadIdx.x; q < (int)(sizeof(JxbSimArgs) / 8); q += blockDim.x) dst[q] = src[q];
    __syncthreads();
    item_idx = mi.y;
    return s;
  }
  return L;
}

// MINB CTAs of NT threads per SM: float by default at most 64 registers, so that two
// 512-thread CTAs (four of 256) fit an SM; the wide variant (JxbSimArgs.wide) of the
// 256-thread kernels allows 128 registers with two CTAs per SM.
template <typename T, int NT>
constexpr int kMinBlocks = sizeof(T) == 4 ? 1024 / NT : 1;

template <typename T, int NT, int MINB, bool GM, bool MULTI>
__global__ void __launch_bounds__(NT, MINB) sim_forward_kernel(JxbSimArgs L) {
  extern __shared__ __align__(16) char smem_raw[];
  int item_idx;
  const JxbSimArgs& a = item_args<T, MULTI>(L, item_idx);
  sim_forward_body<T, GM>(a, L, item_idx, smem_raw);
}

template <typename T, int NT, int MINB, bool GM, bool MULTI>
__global__ void __launch_bounds__(NT, MINB) sim_backward_kernel(JxbSimArgs L) {
  extern __shared__ __align__(16) char smem_raw[];
  int item_idx;
  const JxbSimArgs& a = item_args<T, MULTI>(L, item_idx);
  sim_backward_body<T, GM>(a, L, item_idx, smem_raw);
}

// One instantiation of the forward or adjoint kernel for a launch shape.
typedef void (*SimKernel)(JxbSimArgs);

// Defined by the instantiation units (jxb_sim_inst.cu): the kernel of element type
// T (0 float, 1 double), kind (0 forward, 1 adjoint) and CTA size class NT
// (256, 512, 1024) for global work areas (gm) and multi-request launches (multi);
// `wide` selects the two-CTAs-per-SM float kernels of up to 256 threads (null where
// there is none).
SimKernel sim_kernel_f32_fwd_256(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f32_fwd_512(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f32_fwd_1024(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f32_bwd_256(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f32_bwd_384(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f32_bwd_512(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f32_bwd_1024(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f64_fwd_256(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f64_fwd_512(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f64_fwd_1024(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f64_bwd_256(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f64_bwd_512(bool gm, bool multi, bool wide);
SimKernel sim_kernel_f64_bwd_1024(bool gm, bool multi, bool wide);

}  // namespace jxb
