/*
 * jxb.h - C ABI of libjxb, the sm_100a kernels behind jaxley_pytorch_b200.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream, returns an
 * int status (JXB_OK = 0) and never allocates device memory; buffers are owned by the
 * caller. The ABI replaces these reference interfaces of jaxley-pytorch:
 *
 *   jxb_tree_solve_registers  <- kernels/tree_solve.py:228-287 (_tree_solve_kernel),
 *                                launched by TreeSolveKernel.solve, :396-422, and the
 *                                custom op jaxley_pytorch::tree_solve, :518-563
 *   jxb_tree_solve_levels     <- kernels/tree_solve.py:290-375 (_tree_solve_levels_kernel),
 *                                launched by _launch_levels, :467-482, and the custom
 *                                op jaxley_pytorch::tree_solve_levels, :589-609
 *   jxb_synapse_forward       <- kernels/synapse_step.py:121-182 (_forward_kernel) and
 *                                the op jaxley_pytorch::synapse_step, :336-363
 *   jxb_synapse_backward      <- kernels/synapse_step.py:184-305 (_backward_kernel) and
 *                                :307-330 (_presynaptic_sum_kernel), the op
 *                                jaxley_pytorch::synapse_step_backward, :372-416
 *   jxb_sim_forward           <- the per-step body of jx.integrate: integrate.py:624-636
 *                                -> Module._step_with_plan, modules/base.py:3214-3400
 *                                (channels :3402-3542, voltage solve
 *                                solver_voltage.py:294-359), fused into one launch per
 *                                segment of steps
 *   jxb_sim_backward          <- loss.backward() through the same loop: the autograd
 *                                of _step_with_plan and _DHSSolve.backward,
 *                                solver_voltage.py:143-187, with the time
 *                                checkpointing of utils/torch_utils.py:141-198
 */
#ifndef JXB_H_
#define JXB_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  JXB_OK = 0,
  JXB_ERR_ARG = 1,        /* bad pointer, size or shape */
  JXB_ERR_DTYPE = 2,      /* dtype not float32/float64 */
  JXB_ERR_SMEM = 3,       /* the work item does not fit in shared memory */
  JXB_ERR_LAUNCH = 4,     /* the CUDA launch failed (see jxb_last_error) */
  JXB_ERR_TOO_LARGE = 5   /* a tree is larger than the selected kernel supports */
};

enum { JXB_F32 = 0, JXB_F64 = 1 };

/* ---------------------------------------------------------------------------------
 * Tree solve: x = A^{-1} s for a forest, A[i,i] = d[i], A[i,p] = l[i], A[p,i] = u[i]
 * (p = parent of i), batch-major arrays of shape (batch, n).
 * ------------------------------------------------------------------------------- */

/* Schedule of the level variant: whole trees packed into blocks; inside a block the
 * nodes are grouped into chains (a node and its only child form one chain), chains
 * are ordered by level (leaf chains first). Node indices are solve-order indices of
 * the caller's arrays; `perm` lists the block's nodes in chain order. */
typedef struct {
  int32_t n_nodes;        /* nodes per batch row */
  int32_t n_blocks;
  int32_t max_block_nodes;
  int32_t max_levels;
  const int32_t* block_info;  /* (n_blocks, 4): node start, node count, chain start, level-ptr start */
  const int32_t* block_levels;/* (n_blocks,) number of chain levels */
  const int32_t* perm;        /* (n_nodes,) chain-order position -> node index (absolute) */
  const int32_t* chain_top;   /* (n_chains,) first node (chain-order position, block-relative) */
  const int32_t* chain_len;   /* (n_chains,) */
  const int32_t* chain_ptop;  /* (n_chains,) parent of the top (block-relative) or -1 */
  const int32_t* chain_cptr;  /* (n_chains+1,) child chains: CSR into chain_child */
  const int32_t* chain_child; /* tops of the child chains (block-relative) */
  const int32_t* level_ptr;   /* per block (levels+1) chain offsets */
} JxbTreeSchedule;

int jxb_tree_solve_levels(int dtype, const void* d, const void* l, const void* u,
                          const void* s, void* x, int64_t batch,
                          const JxbTreeSchedule* sched, void* stream);

/* Register variant: every block of whole trees of at most 32 * regs_per_lane nodes
 * is held in registers for one batch row. Up to 256 nodes (regs_per_lane <= 8) one
 * warp solves it with warp shuffles for the parent/child exchanges; from 512 to 8192
 * nodes (regs_per_lane 16 .. 256) a CTA of 4 * regs_per_lane threads, 8 nodes a
 * thread, exchanges through shared memory. */
typedef struct {
  int32_t n_nodes;
  int32_t n_blocks;
  int32_t regs_per_lane;      /* power of two, 1 .. 256: block width / 32 */
  int32_t num_slots;          /* max children per node */
  const int32_t* block_info;  /* (n_blocks, 4): start, length, height, depth of the block */
  const int32_t* rel_parent;  /* (n_blocks, 32*regs) parent (block-relative), self for roots */
  const int32_t* rel_height;  /* (n_blocks, 32*regs) height, -1 for padding */
  const int32_t* rel_depth;   /* (n_blocks, 32*regs) depth, -1 for padding */
  const int32_t* rel_children;/* (n_blocks, num_slots, 32*regs) children or -1 */
} JxbRegSchedule;

int jxb_tree_solve_registers(int dtype, const void* d, const void* l, const void* u,
                             const void* s, void* x, int64_t batch,
                             const JxbRegSchedule* sched, void* stream);

/* ---------------------------------------------------------------------------------
 * Fused simulation step (bwd_euler + DHS) over segments of steps.
 * ------------------------------------------------------------------------------- */

typedef struct {
  int32_t node0, n_nodes;     /* internal node range of the block */
  int32_t slot0, n_slots;     /* state-slot range */
  int32_t chain0, n_chains;   /* chains of the block, sorted by level */
  int32_t level0, n_levels;   /* level_ptr[level0 .. level0 + n_levels] */
  int32_t pslot0, n_pslots;   /* parameter-slot range */
  int32_t n_gslots, pad1;     /* gradient slots of the block (adjoint sizing) */
} JxbBlock;

typedef struct {
  int32_t block;              /* index into blocks */
  int32_t row0, n_rows;       /* batch rows of the state buffer */
  int32_t pad;
} JxbItem;

typedef struct JxbSimArgs_ {
  int32_t dtype;
  int32_t batch;              /* rows of state / pscale / rec buffers */
  int32_t n_nodes, n_slots, n_pslots, n_cols;
  int32_t n_items, n_steps;   /* steps in this launch */
  int32_t t0;                 /* absolute index of the first step */
  int32_t max_rows;           /* rows per item (shared-memory sizing) */
  int32_t max_nodes, max_slots;   /* largest block: nodes, state slots */
  int32_t max_chains, max_child;  /* largest block: chains, child-chain links */
  int32_t max_levels, max_pslots; /* largest block: chain levels, parameter slots */
  int32_t threads, pad3;          /* threads per CTA (0 = default) */
  double dt;
  /* topology, internal (chain) node order */
  const int32_t* node_class;  /* (n_nodes,) */
  const int32_t* soff;        /* (n_nodes+1,) state-slot offsets */
  const int32_t* poff;        /* (n_nodes,) first parameter slot (runs may be shared) */
  const void* a_low;          /* (n_nodes,) axial conductance row i -> parent */
  const void* a_up;           /* (n_nodes,) axial conductance parent row -> i */
  const void* gsum;           /* (n_nodes,) sum of axial conductances sinking into i */
  const void* cm;             /* (n_nodes,) capacitance */
  const int32_t* cls_ptr;     /* (n_classes+1,) entries of every node class */
  const int32_t* cls_comp;    /* (n_classes,) 1 for compartments, 0 for branchpoints */
  const int32_t* cls_prog;    /* (n_classes,) compile-time program id, 0 = interpreted */
  const void* entries;        /* channel entries (16-bit fields, see jxb_channels.cuh) */
  int32_t n_classes, n_entries;
  const void* pbase;          /* (n_pslots,) */
  const int32_t* pcol;        /* (n_pslots,) column of pscale, 0 = no scale */
  const void* pscale;         /* (batch, n_cols); column 0 holds 1 */
  const JxbBlock* blocks;
  const JxbItem* items;
  const int32_t* chain_top;   /* internal node index */
  const int32_t* chain_len;
  const int32_t* chain_ptop;  /* internal node index or -1 */
  const int32_t* chain_cptr;
  const int32_t* chain_child; /* internal node index of child-chain tops */
  const int32_t* level_ptr;   /* chain offsets relative to the block's chain0 */
  const int32_t* gk;          /* (n_pslots,) gradient rank of a trainable parameter, -1 */
  const int32_t* gbase;       /* (n_nodes,) first gradient slot of a node in its block */
  int32_t max_gslots;         /* largest number of gradient slots of a block */
  int32_t wide;               /* float, up to 256 threads, not multi: kernels for two CTAs
                                 per SM with up to 128 registers a thread (default: four
                                 CTAs with 64) */
  const int32_t* parent;      /* (n_nodes,) parent (internal order) or -1 */
  const int32_t* kid_ptr;     /* (n_nodes+1,) children CSR */
  const int32_t* kid;         /* children (internal order) */
  /* stimulus: i_ext[node] += stim[t][b][idx] / area[node] * 1e5 */
  const int32_t* stim_ptr;    /* (n_nodes+1,) CSR over nodes */
  const int32_t* stim_idx;
  const void* area;           /* (n_nodes,) */
  const void* stim;           /* (stim_steps, stim_rows, n_stim) */
  int32_t n_stim, stim_steps, stim_rows, pad0;
  /* synaptic terms added to lin/const before dividing by cm (may be null) */
  const void* syn_lin;        /* (batch, n_nodes) */
  const void* syn_const;      /* (batch, n_nodes) */
  /* recordings: CSR over nodes */
  const int32_t* rec_ptr;     /* (n_nodes+1,) */
  const int32_t* rec_slot;    /* node-relative slot, -1 records 0 */
  const int32_t* rec_col;     /* output column */
  void* rec_out;              /* (T + 1, batch, n_rec), time index t0 + step + 1 */
  int32_t n_rec, pad1;
  /* state */
  void* state;                /* (batch, n_slots), updated in place */
  void* ckpt;                 /* optional (n_ckpt, batch, n_slots): state at t0 + m*ckpt_every */
  int32_t ckpt_every, ckpt_base;  /* ckpt index of t0 is (t0 - ckpt_base) / ckpt_every */
  /* Trajectory. Adjoint: scratch (n_steps, batch, n_slots) for the state before each
   * recomputed step and (n_steps, batch, n_nodes) for the reciprocal pivots; with
   * traj_stored the caller's forward has filled both and the adjoint reads them
   * (traj then holds n_steps + 1 entries, the last being the state after the
   * segment, and ckpt must point at entry 0). Forward (optional, mode 0): the launch
   * stores the state before each of its steps and after its last step
   * (n_steps + 1 entries) and, with traj_piv, the pivots of each step. */
  void* traj;
  void* traj_piv;
  /* adjoint */
  void* adj;                  /* (batch, n_slots) adjoint of the state, updated in place */
  const void* rec_grad;       /* (T + 1, batch, n_rec) gradient of the recordings */
  double* pgrad;              /* (batch, n_cols) float64, accumulated: d loss / d pscale */
  int32_t mode;               /* 0 = step, 1 = initial currents only */
  int32_t traj_stored;        /* adjoint: traj / traj_piv hold the forward's values */
  /* Optional work areas in global memory instead of shared memory, for blocks whose
   * working set exceeds the shared memory of a CTA: item i uses the bytes
   * [gscratch + i * gscratch_stride, + gscratch_stride). gscratch is 256-byte aligned
   * and gscratch_stride a multiple of 256 of at least jxb_sim_smem_bytes(args, kind).
   * Null: the work areas live in shared memory. */
  void* gscratch;
  int64_t gscratch_stride;
  /* Optional node schedule of the per-node phases (channels, adjoint): for block b,
   * sched[sched_ptr[b] .. sched_ptr[b+1]) holds sched_warps x k x 32 block-relative
   * node indices (-1 = idle lane): warp w, iteration q, lane l processes
   * sched[sched_ptr[b] + (w * k + q) * 32 + l]. Used when sched_warps equals the
   * launch's warps per CTA; otherwise (or null) nodes are strided over the threads. */
  const int32_t* sched_ptr;
  const int16_t* sched;
  int32_t sched_warps, pad5;
  /* Optional (adjoint): the per-node gradient slots of item i in global memory at
   * [gacc + i * gacc_stride, + max_rows * max_gslots * sizeof(dtype)) instead of
   * shared memory (frees shared memory for more CTAs per SM). 256-byte aligned,
   * stride a multiple of 256. Null: the slots live in shared memory. */
  void* gacc;
  int64_t gacc_stride;
  /* Set by jxb_sim_forward_multi / jxb_sim_backward_multi (leave null): the device
   * copies of the requests' arguments and the (request, item) pair of every CTA. */
  const struct JxbSimArgs_* multi;
  const int32_t* multi_items;
  /* Synapse outputs by target (optional; needs syn_lin/syn_const): with syn_ptr set,
   * syn_lin/syn_const hold the synapse step's per-target slope and offset of every
   * synapse type (the `lin`, `const` outputs of jxb_synapse_forward, concatenated),
   * and node i (internal order) adds, for q in [syn_ptr[i], syn_ptr[i+1]) and row b,
   * lin += syn_lin[syn_off[q] + b * syn_rs[q]] and const -= syn_const[...], as the
   * reference's index_add of (lin, -const) (modules/network.py:402-407). The adjoint
   * then writes d loss / d syn_lin and d loss / d syn_const of its step to
   * g_syn_lin / g_syn_const at the same positions. */
  const int32_t* syn_ptr;
  const int32_t* syn_off;
  const int32_t* syn_rs;
  void* g_syn_lin;
  void* g_syn_const;
  /* Clamps (optional; modules/base.py:3305-3308 and :3396-3398, fed by data_clamps /
   * Module.clamp, integrate.py:345-375): for q in [clamp_ptr[i], clamp_ptr[i+1]) of
   * node i (internal order), after step t the node's state slot clamp_slot[q]
   * (node-relative) takes clamp[t][b][clamp_col[q]] (the row index b is 0 when
   * clamp_rows is 1). Slot 0 (v) is set after the voltage solve; the node's last slot
   * then receives the solve output before the clamp, which the adjoint reads. Other
   * slots are set after the step's channel update, after the currents were taken.
   * Entries of one node apply in order (the last wins). The adjoint drops the
   * gradient of every clamped value. */
  const int32_t* clamp_ptr;   /* (n_nodes+1,) or null */
  const int32_t* clamp_slot;
  const int32_t* clamp_col;
  const void* clamp;          /* (clamp_steps, clamp_rows, n_clamp) */
  int32_t n_clamp, clamp_steps, clamp_rows, pad6;
  /* Optional failure flag (device int32, may be null): a launch whose final states
   * (forward) or state adjoints and parameter gradients (adjoint) hold a value that is
   * not finite ORs JXB_NONFINITE into it; an adjoint launch whose bounded wait for
   * a bulk copy gave up ORs JXB_TIMEOUT (its results are then invalid). The host reads
   * and clears it between launches; the kernels never stop or fault on either. */
  int32_t* status;
  /* Step scheme of the voltage (modules/base.py:3327-3365): JXB_SCHEME_BWD_EULER, or
   * JXB_SCHEME_CN (Crank-Nicolson: the implicit system of half a step, then
   * v' = 2 v_half - v; the channels step by the whole dt in both). */
  int32_t scheme, pad7;
} JxbSimArgs;

enum { JXB_NONFINITE = 1, JXB_TIMEOUT = 2 };
enum { JXB_SCHEME_BWD_EULER = 0, JXB_SCHEME_CN = 1 };

int jxb_sim_forward(const JxbSimArgs* args, void* stream);
int jxb_sim_backward(const JxbSimArgs* args, void* stream);

/* jxb_sim_backward without caller scratch: no counterpart in the reference. For
 * callers that cannot allocate device memory during the simulation (buffers handed
 * over from a host-owned memory pool, or a plugin whose framework allocator must not
 * be re-entered from a step). The trajectory scratch (args->traj, args->traj_piv are
 * ignored) lives in a fixed 32 MiB device array of the library, held by every GPU
 * that loads it until exit; segments needing more return JXB_ERR_TOO_LARGE. The first
 * call on a device (and the first after that device's context was reset) looks up the
 * array's device address (cudaGetSymbolAddress) with that device current and should
 * come before any stream capture; the look-up is guarded for calls from several host
 * threads. All calls share the
 * array: calls that overlap on the GPU (other streams, other threads) race. Nothing
 * in the array needs to start at zero: every slot a segment reads was written earlier
 * in the same launch. It calls no cudaMalloc, cudaFree or allocating library routine. */
int jxb_sim_backward_noalloc(const JxbSimArgs* args, void* stream);

/* Forward-mode derivatives: a forward launch (mode 0, 1 or 2) in dual numbers. Every
 * floating-point array of `args` (a_low, a_up, gsum, cm, pbase, pscale, area, stim,
 * clamp, state, rec_out, ckpt) holds (value, tangent) pairs of the element type
 * `dtype`, interleaved and aligned to the pair size (8 or 16 bytes); the launch
 * advances both, so that the tangents of the states and recordings are the
 * directional derivatives along the inputs' tangents. Replaces the reference's
 * forward-mode rule of the tree solve inside a forward-AD level (_DHSSolveForwardAD,
 * solver_voltage.py:190-224; dhs_solve, :235-236) for the fused step. Trajectory
 * stores, synapse inputs and multi-request launches are not taken (traj, traj_piv,
 * syn_lin, syn_const and multi must be null). Up to 512 threads. */
int jxb_sim_tangent(const JxbSimArgs* args, void* stream);
int64_t jxb_sim_tangent_smem_bytes(const JxbSimArgs* args);
int64_t jxb_sim_smem_bytes(const JxbSimArgs* args, int backward);

/* Continuous batching of requests (no counterpart in the reference, whose
 * `jx.integrate` simulates one module per call, integrate.py:396-666): one launch
 * runs the work items of several independent problems. `launch` gives the
 * work-area sizing (max_* fields at least each request's, n_entries and n_classes
 * at least each request's, max_gslots for the adjoint), threads, and optional
 * gscratch / gacc buffers indexed by the launch's CTA; `reqs` (host, n_reqs) are the
 * requests' arguments as for jxb_sim_forward / jxb_sim_backward, each with its own
 * state, time window (t0, n_steps), buffers and items; `pairs` (host, n_pairs x 2)
 * the (request, item) pair of every CTA. The library validates every request and
 * pair, copies them into `dev_scratch` (device, 256-byte aligned, at least
 * jxb_sim_multi_scratch_bytes bytes) on `stream` and launches. The scratch must
 * stay untouched until the launch has run. */
int jxb_sim_forward_multi(const JxbSimArgs* launch, const JxbSimArgs* reqs, int n_reqs,
                          const int32_t* pairs, int n_pairs, void* dev_scratch, int64_t scratch_bytes,
                          void* stream);
int jxb_sim_backward_multi(const JxbSimArgs* launch, const JxbSimArgs* reqs, int n_reqs,
                           const int32_t* pairs, int n_pairs, void* dev_scratch, int64_t scratch_bytes,
                           void* stream);
int64_t jxb_sim_multi_scratch_bytes(int n_reqs, int n_pairs);

/* ---------------------------------------------------------------------------------
 * Synapses in the regular layout (E = T * k synapses ordered by target).
 * ------------------------------------------------------------------------------- */
typedef struct {
  int32_t dtype, model;       /* 0 KineticSynapse, 1 SigmoidRateSynapse */
  int32_t batch, n_nodes, n_syn, k;
  int32_t targets_are_nodes, store_current;
  const void* v;              /* (batch, n_nodes) */
  const void* s;              /* (batch, n_syn) kinetic state or null */
  const int32_t* pre;         /* (n_syn,) */
  const int32_t* targets;     /* (n_syn / k,) */
  const void* p[6];           /* (n_syn,) parameters in the reference order */
  const void* area;           /* (n_syn,) area of the postsynaptic compartment */
  const void* scalars;        /* (2,) dt, diff */
  void* s_new;                /* (batch, n_syn) or null */
  void* current;              /* (batch, n_syn) or null */
  void* lin;                  /* (batch, n_syn / k) */
  void* cst;                  /* (batch, n_syn / k) */
  /* backward */
  const void* g_s_new;        /* (batch, n_syn) or null */
  const void* g_current;      /* (batch, n_syn) or null */
  const void* g_lin;          /* (batch, n_syn / k) */
  const void* g_const;        /* (batch, n_syn / k) */
  void* g_s;                  /* (batch, n_syn) or null */
  void* g_v;                  /* (batch, n_nodes), overwritten */
  void* g_params;             /* (n_need, n_syn), overwritten */
  void* g_pre;                /* (n_syn, batch) scratch for the presynaptic sum */
  void* g_post;               /* (batch, n_syn / k) scratch for the postsynaptic sum */
  int32_t need;               /* bit mask of parameters that need gradients */
  int32_t inv_width, n_pre_nodes;
  int32_t accumulate;         /* 0: g_v and g_params are overwritten (the op); 1: the step's
                                 voltage gradient is added to g_v (presynaptic and target
                                 nodes) and its parameter gradients to g_params, as an adjoint
                                 that sums over steps does; g_post is then unused */
  const int32_t* inv;         /* (n_pre_nodes, inv_width) synapses of every pre node */
  const int32_t* pre_nodes;   /* (n_pre_nodes,) */
} JxbSynArgs;

int jxb_synapse_forward(const JxbSynArgs* args, void* stream);
int jxb_synapse_backward(const JxbSynArgs* args, void* stream);

/* Text of the last error of this thread (static storage). */
const char* jxb_last_error(void);
int jxb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* JXB_H_ */
