/*
 * flyb200 -- C ABI of the B200-native brain-step engine.
 *
 * Every entry point takes plain pointers and sizes, launches on the caller's CUDA stream
 * (`stream` is a cudaStream_t passed as void*), allocates nothing, and returns 0 or a
 * cudaError_t / FLYB_E* code. Device buffers are owned by the caller (in the Python host
 * layer: torch tensors). All kernels are compiled for sm_100a only. Column / weight / edge
 * arrays of a sparse matrix may be null when the matrix has no entries.
 *
 * Two groups of entry points:
 *
 *  1. Reference-compatible launchers. Same names, argument order, pointer order and
 *     semantics as the ctypes-bound functions of flyverse/kernels/neural.cu, so the
 *     reference's loader (flyverse/cuda.py:37-79) can bind this library unchanged.
 *
 *  2. The native path: a fused, event-driven LIF step over an exact integer delay ring,
 *     the fused optic-lobe SpMV/SpMM substep, the held-input products, the optic adjoint,
 *     and the readout / photoreceptor stages. State is laid out neuron-major, fly-minor:
 *     element (neuron i, fly b) of a (B, N) state lives at [i * batch + b].
 */
#ifndef FLYB200_H
#define FLYB200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define FLYB_OK              0
#define FLYB_EINVAL          1001   /* bad size, null pointer or inconsistent arguments */
#define FLYB_EBARRIER        1002   /* a bounded grid-barrier wait gave up (see status word) */
#define FLYB_ECOOP           1003   /* persistent launch does not fit co-resident on the device */
#define FLYB_ETOOBIG         1004   /* request exceeds a stated maximum */

/* ================================================================== 1. reference-compatible
 * Pointer arrays and flags exactly as flyverse/cuda.py builds them.                        */

/* Fused LIF update, one step, batch-major (B, N) float32 state.
 * Replaces flyverse/kernels/neural.cu:54 `launch_lif` (pointer order cuda.py:103-107:
 * v, g, drive, adapt, refrac, active, prob, rnd, res, std_u, spikes, out, rate, counts, P, phase;
 * flags 1 Poisson, 2 STD, 4 counts, 8 adapt, 16 per-phase coefficients (8, N), 32 skip frozen). */
int launch_lif(void** p, int n, int batch, int flags, void* stream);

/* dr = clip01(v + b) - b.  Replaces neural.cu:80 `launch_optic_dr` (p: v, b, dr). */
int launch_optic_dr(void** p, int n, int batch, void* stream);

/* Optic substep update.  Replaces neural.cu:84 `launch_optic`
 * (p: v, adapt, dr, y, pr, spk, a, b; cuda.py:123-128). */
int launch_optic(void** p, int n, int batch, float gr, float ga, float aad, void* stream);

/* out(batch, rows) = x(batch, cols) @ CSR^T, fp32 or fp16 weights.
 * Replaces neural.cu:105 `launch_csr` (p: ptr, idx, w, x, out; cuda.py:151-152). */
int launch_csr(void** p, int rows, int cols, int batch, int half, void* stream);

/* g(batch, n) += x(batch, n) scattered over CSC columns (float atomics, as the reference).
 * Replaces neural.cu:124 `launch_events` (p: ptr, idx, w, x, g, pre_ids; cuda.py:167-168). */
int launch_events(void** p, int n, int batch, int half, int count, void* stream);

/* out[b*stride + k] = mean of rates[b, idx[ptr[k]:ptr[k+1]]] in fixed-order double.
 * Replaces neural.cu:141 `launch_means` (p: ptr, idx, rates, out; cuda.py:180). */
int launch_means(void** p, int n, int groups, int batch, int stride, void* stream);

/* ================================================================== 2. native path */

/* LIF flags */
#define FLYB_LIF_POISSON      1    /* Poisson forcing from poisson_p                          */
#define FLYB_LIF_STD          2    /* short-term depression (transmit spike * res)            */
#define FLYB_LIF_COUNTS       4    /* spike_counts += spikes                                  */
#define FLYB_LIF_ADAPT        8    /* adaptation current                                      */
#define FLYB_LIF_EXT_UNIFORM  16   /* Poisson uniforms from `uniforms` instead of Philox      */
#define FLYB_LIF_SKIP_FROZEN  32   /* frozen cells at rest are left untouched                 */
#define FLYB_LIF_EPISODES     64   /* per-fly remaining-step counters gate the update         */
#define FLYB_LIF_DEFER_DELIVERY 256 /* per-step launches (register or staged path): the update
                                      kernel lists the transmitting items (one entry per 1024
                                      out-edges) in `spike_list` and a second kernel delivers
                                      them, one block per entry; needs spike_list / spike_n /
                                      spike_cap                                                */
#define FLYB_LIF_NO_ADVANCE   128  /* leave `clock` and `fly_steps` as they are: other launches of
                                      the same steps cover the other neurons; flyb_lif_advance
                                      moves them on once all have run                           */
#define FLYB_LIF_PULL_DELIVERY 512 /* per-step launches (register or staged path), count ring,
                                      batch a multiple of 32 (at most 256), raster on: the
                                      update kernels only record the step's spikes in the raster,
                                      then each postsynaptic row sums count x spike over its
                                      inputs (pull_ptr / pull_pre / pull_meta) into the write
                                      slot, the same exact integers the scatter adds. A launch
                                      over all neurons pulls after every step; launches over
                                      neuron ranges leave it to flyb_lif_pull                    */

/* Delay-ring element types */
#define FLYB_RING_COUNT  0   /* int32 signed synapse counts; g += w_syn * count (exact sum)     */
#define FLYB_RING_FIXED  1   /* int64 Q32.32 millivolts; each edge rounds w*x once (exact sum)  */

/* Launch modes */
#define FLYB_LAUNCH_STEP       0   /* one kernel launch per step (the "plain" kernel)        */
#define FLYB_LAUNCH_PERSISTENT 1   /* one cooperative launch for all steps, grid barrier/step */

#define FLYB_SLOW_MAX_CLASSES 2   /* slow receptor classes: classical metabotropic, monoamine */

/* LIF coefficient vector P[FLYB_LIF_NPARAM] (float32) */
enum {
  FLYB_P_V_REST = 0, FLYB_P_V_RESET, FLYB_P_V_TH, FLYB_P_A_M, FLYB_P_A_S, FLYB_P_DT,
  FLYB_P_T_REF, FLYB_P_ADAPT_JUMP, FLYB_P_A_AD, FLYB_P_A_STD, FLYB_P_A_R, FLYB_P_RATE_GAIN,
  FLYB_P_W_SYN, FLYB_LIF_NPARAM
};

/* Words of caller scratch a persistent LIF launch needs (grid-barrier counters). */
#define FLYB_LIF_SYNC_WORDS 64

typedef struct flyb_lif_args {
  int n;                 /* neurons                                                  */
  int batch;             /* flies                                                    */
  int n_delay;           /* D: a spike of step t is delivered at step t + D          */
  int ring_slots;        /* R >= D + 1 ring slots                                    */
  int ring_mode;         /* FLYB_RING_COUNT or FLYB_RING_FIXED                       */
  int ring_pos;          /* slot read by the first step                              */
  int flags;             /* FLYB_LIF_*                                               */
  int nsteps;            /* steps to run                                             */
  int launch;            /* FLYB_LAUNCH_*                                            */
  int block;             /* threads per block (multiple of 32; 0 = default 256)       */
  int grid;              /* persistent grid size cap (0 = all co-resident blocks)    */
  int raster_slots;      /* 0: raster is [nsteps][words]; else a ring of that many slots */
  int raster_pos;        /* ring slot written by the first step (raster_slots > 0)   */
  int fly0;              /* global index of local fly 0 (Philox key when flies are sharded) */
  int items_per_thread;  /* 0 auto (4 when aligned), 1, 2 or 4 consecutive items per thread */
  int staged;            /* per-step launches only: 1 stages each block's state chunks through
                            shared memory with bulk async copies, the next chunk loading while
                            the current one is updated and delivered (needs the items of the
                            launch, n_count * batch, and n_first * batch to be multiples of 4
                            and 16-byte aligned arrays; otherwise the register path runs) */
  int n_first;           /* update neurons [n_first, n_first + n_count) only (n_count 0: to
                            the end); n_first * batch must be a multiple of 32. Their spikes
                            are delivered to every postsynaptic neuron as usual; the state
                            of the other neurons is not touched */
  int n_count;
  long long step0;       /* global step index of the first step (Philox counter)     */
  unsigned long long seed;
  /* outgoing synapses, pre-major (CSC of W[post, pre]) */
  const int* out_ptr;    /* [n + 1]                                                  */
  const int* out_edge;   /* [nnz][2]: {post, count} (COUNT) or {post, float bits of w} (FIXED) */
  /* state, [n][batch] float32 */
  float* v; float* g; float* refrac; float* adapt; float* res;
  float* rate; float* counts; float* spikes;
  const float* drive; const float* poisson_p;
  const float* active;   /* [n] 1 = spiking, 0 = frozen                              */
  const float* std_u;    /* [n] depression use fraction                              */
  const float* params;   /* [FLYB_LIF_NPARAM] host memory                            */
  void* ring;            /* [R][n][batch] int32 (COUNT) or int64 (FIXED)             */
  const float* uniforms; /* [nsteps][n][batch] when FLYB_LIF_EXT_UNIFORM             */
  int* fly_steps;        /* [batch] remaining steps per fly when FLYB_LIF_EPISODES: fly b
                            is live for local steps k < fly_steps[b]; after the run each
                            entry is lowered by the steps taken (never below 0)      */
  long long* clock;      /* optional device [3]: {step, ring_pos, raster_pos}. When set it
                            replaces step0 / ring_pos / raster_pos and the launch advances
                            it by nsteps, so a captured CUDA graph replays correctly */
  unsigned* raster;      /* optional spike bits, words of ceil(n*batch/32), bit i*batch+b:
                            [nsteps][words], or [raster_slots][words] used as a ring   */
  unsigned long long* events; /* optional [1]: += synaptic events (edges delivered)    */
  int* status;           /* [4] device words: [0] error code, [1] where, [2] step    */
  int* sync;             /* [FLYB_LIF_SYNC_WORDS] zeroed device scratch (persistent) */
  void* spike_list;      /* FLYB_LIF_DEFER_DELIVERY: [spike_cap] int4 entries (device)  */
  unsigned* spike_n;     /* FLYB_LIF_DEFER_DELIVERY: one device word (reset each step)  */
  long long spike_cap;   /* entries spike_list holds: flyb_lif_spike_capacity(a) or more */
  const float* adapt_jump; /* optional [n]: per-neuron adaptation jump (mV per spike) under
                            FLYB_LIF_ADAPT, the reference's adapt_by_type (brain.py:497-506);
                            null = params[FLYB_P_ADAPT_JUMP] for every neuron             */
  /* Per-neuron clocks (Brain.set_clocks, brain.py:618-640 and the clocked step :899-957): neuron
   * i integrates only on steps with step % clock_k[i] == 0, with the coefficients of a step of
   * clock_k[i] * dt; its synaptic input arriving in between is held in clock_acc and applied on
   * its next update. Null clock_k: every neuron every step. Runs one launch per step (launch,
   * items_per_thread, staged are ignored); FLYB_LIF_DEFER_DELIVERY is not allowed with it. */
  const unsigned char* clock_k; /* [n] update period in steps, 1..255 (device)               */
  const float* clock_coef; /* [max period + 1][FLYB_CLOCK_NCOEF] (device): row p holds the
                            coefficients of an update of a period-p neuron, row 0 those of a
                            step on which a neuron does not update                         */
  void* clock_acc;       /* [n][batch] int64 (device): pending input of neurons with period
                            > 1, in ring units (counts, or Q32.32 mV)                       */
  void* slow_clock_acc[FLYB_SLOW_MAX_CLASSES]; /* clocks with the slow tone: [n][batch] int64
                            Q32.32 per class (device), slow input pending at period > 1       */
  /* Slow receptor tone (receptor_model "full": brain.py:551-585, the step :829-845): per class c
   * < slow_classes a tone slow_g[c] (mV) decays by slow_decay[c] per step and takes the delayed
   * input of its own synapse list (pre-major like out_ptr / out_edge, {post, float bits of w}),
   * summed exactly on its own Q32.32 ring; g_slow = sum over classes acts by slow_mode: added to
   * the membrane target, scaling the fast input by clamp(1 + g_slow / slow_norm, slow_clip_lo,
   * slow_clip_hi), or lowering the threshold by min(g_slow, slow_th_max). Runs one launch per step
   * like the clocks. With clocks (the reference's clocked step) a class decays by column
   * FLYB_CLOCK_A_SLOW0 + c of the neuron's phase row instead of slow_decay[c], and its input to a
   * neuron with period > 1 waits in slow_clock_acc[c] for the update. slow_classes 0: no tone. */
  int slow_classes;      /* 0..FLYB_SLOW_MAX_CLASSES                                      */
  int slow_mode;         /* FLYB_SLOW_ADDITIVE, FLYB_SLOW_GAIN or FLYB_SLOW_THRESHOLD      */
  float slow_norm, slow_clip_lo, slow_clip_hi, slow_th_max;
  float slow_decay[FLYB_SLOW_MAX_CLASSES];
  const int* slow_out_ptr[FLYB_SLOW_MAX_CLASSES];   /* [n+1] per class (device)          */
  const int* slow_out_edge[FLYB_SLOW_MAX_CLASSES];  /* [nnz][2] per class (device)       */
  void* slow_ring[FLYB_SLOW_MAX_CLASSES];           /* [R][n][batch] int64 per class     */
  float* slow_g[FLYB_SLOW_MAX_CLASSES];             /* [n][batch] tone per class (mV)    */
  float* g_slow;                                    /* [n][batch] summed tone (mV)       */
  /* FLYB_LIF_PULL_DELIVERY: the inputs of each neuron (rows of W[post, pre]) in chunks of 32
   * entries: pull_ptr [n+1] first chunk of each row, pull_meta [chunks] = (base << 5) | planes:
   * entry l of the chunk carries count base + d_l, 0 <= d_l < 2^planes. Two table formats:
   * pull_nplanes = 0 (packed, planes <= 8, n < 2^24): pull_pre [chunks][32] = pre | d_l << 24,
   * 0xFFFFFF padding a row's last chunk, pull_planes unused (may be null);
   * pull_nplanes = 16: pull_pre [chunks][32] presynaptic neuron (-1 padding) and pull_planes
   * [chunks][16] the d_l as bit planes (bit l of plane p = bit p of d_l), 16-byte aligned.
   * The update kernels record each step's spike words in pull_bits as well, and pulls deliver
   * groups of pull_group consecutive steps at once: one gather per input then fetches the input's
   * words of every step of the group (one 32-byte sector when pull_group = 8 / (batch / 32)). */
  const int* pull_ptr;
  const int* pull_pre;
  const unsigned* pull_planes;
  int pull_nplanes;
  const int* pull_meta;
  int pull_group;        /* L: 1, or 8 / (batch / 32) when 2 L <= n_delay                       */
  int pull_steps;        /* flyb_lif_pull: undelivered steps to deliver now, 1..L               */
  int pull_phase;        /* runs over all neurons: (index of the first step) mod L; they pull
                            at every group end and after their last step                       */
  unsigned* pull_bits;   /* [2][ceil(n * batch / 32)][L] words (device, 32-byte aligned): the
                            spike words of the last two groups, word w of step t at
                            (((t / L) & 1) * words + w) * L + t % L                            */
  long long* pull_state; /* [3] device: {first undelivered step, the ring position of that step,
                            0}; moved on by each pull. It must equal {step, ring position} of the
                            next step to run (step0 / ring_pos, or clock[0] / clock[1]) whenever
                            nothing is pending                                                  */
  int pull_grid;         /* blocks of a pull launch (0: one wave of resident blocks); fewer leave
                            SM room to kernels running beside it on other streams               */
} flyb_lif_args;

/* flyb_lif_args.slow_mode */
enum { FLYB_SLOW_ADDITIVE, FLYB_SLOW_GAIN, FLYB_SLOW_THRESHOLD };

/* Columns of flyb_lif_args.clock_coef */
enum {
  FLYB_CLOCK_A_M, FLYB_CLOCK_A_S, FLYB_CLOCK_DT, FLYB_CLOCK_A_AD, FLYB_CLOCK_A_STD, FLYB_CLOCK_A_R,
  FLYB_CLOCK_RATE_GAIN, FLYB_CLOCK_U, FLYB_CLOCK_POIS, FLYB_CLOCK_A_SLOW0, FLYB_CLOCK_A_SLOW1,
  FLYB_CLOCK_NCOEF
};

int flyb_lif_run(const flyb_lif_args* a, void* stream);

/* FLYB_LIF_PULL_DELIVERY over neuron ranges: delivers the next a->pull_steps undelivered steps
 * (from pull_state, at most pull_group, after every range of those steps ran with
 * FLYB_LIF_NO_ADVANCE) from pull_bits into their write slots, and moves pull_state on. A pull may
 * run on another stream beside the updates of the steps that follow, as long as the update of a
 * step whose words go to the same half of pull_bits (a step of the group after next) and the next
 * pull start only after it; the steps' write slots are read n_delay >= 2 L steps after them.
 * The arguments are those of the launches (any range). No counterpart in the reference (its
 * delivery is a scatter inside the step). */
int flyb_lif_pull(const flyb_lif_args* a, void* stream);

/* Entries a FLYB_LIF_DEFER_DELIVERY step of these arguments can write when every item of the
 * neuron range fires (n_count * batch + batch * out-edges of the range / 1024); reads two row
 * pointers from the device, so call it at set-up, not during stream capture. -1 on bad input. */
long long flyb_lif_spike_capacity(const flyb_lif_args* a);

/* Advance `clock` by a->nsteps and lower `fly_steps` (FLYB_LIF_EPISODES) as the end of a
 * flyb_lif_run does: for runs split over neuron ranges with FLYB_LIF_NO_ADVANCE, after all of
 * them. One small launch on `stream`. No counterpart in the reference (it has one update per step). */
int flyb_lif_advance(const flyb_lif_args* a, void* stream);

/* Deposit transmitted spikes x[n][batch] into ring slot `slot` (checkpoint import of a
 * reference spike buffer). COUNT rings need x in {0, 1}. */
int flyb_ring_deposit(int n, int batch, int ring_mode, const int* out_ptr, const int* out_edge,
                      const float* x, void* ring_slot, void* stream);

/* Optic lobe: `nsteps` fused substeps of y = W_rr @ dr and the rate update, state [m][batch].
 * Substep s reads dr from (s even ? dr : dr_tmp) and writes the next one to the other buffer, so
 * after the call the dr of the final state, clip(v + b, 0, 1) - b, is in `dr` when nsteps is even
 * and in `dr_tmp` when it is odd. */
#define FLYB_OPTIC_HISTORY   1   /* store v and the input of every substep (adjoint recompute)   */
#define FLYB_OPTIC_DR_VALID  2   /* `dr` already holds clip(v + b, 0, 1) - b of the current v (the
                                    final dr of the previous call, buffers swapped by the caller):
                                    the initialisation pass over the state is skipped. Ignored by
                                    flyb_optic_run_noalloc, whose buffers the caller cannot see. */
typedef struct flyb_optic_args {
  int m;                 /* rate units                                               */
  int batch;
  int nsteps;
  int launch;            /* FLYB_LAUNCH_*                                            */
  int block;             /* threads per block (0 = default)                          */
  int grid;              /* persistent grid cap (0 = occupancy)                      */
  int variant;           /* kernel shape: 0 default, 1 / 2 alternatives (autotuned)  */
  int flags;             /* FLYB_OPTIC_*                                             */
  const int* ptr;        /* W_rr CSR row pointers [m + 1], rows = postsynaptic units */
  const int* cw;         /* [nnz][2] interleaved {column, float bits of weight}      */
  const int* rows;       /* optional [m] row order: rows[0, n_long) are long rows, each
                            split across a whole block; the rest one row per warp slot.
                            Null: natural order and n_long = 0                       */
  float* v; float* adapt;                             /* [m][batch]                      */
  float* dr; float* dr_tmp;                           /* [m][batch] ping-pong scratch    */
  const float* pr; const float* spk;                  /* held inputs [m][batch]          */
  const float* a; const float* b;                     /* [m] exp(-dt/tau), operating point */
  float gr, ga, aad;
  int n_long;            /* long rows at the front of `rows`                         */
  float* v_hist;         /* optional [nsteps][m][batch]: v before each substep       */
  float* inp_hist;       /* optional [nsteps][m][batch]: input of each substep       */
  int* status; int* sync;
} flyb_optic_args;

int flyb_optic_run(const flyb_optic_args* a, void* stream);

/* Allocation-free variant of flyb_optic_run; no counterpart in the reference. For callers that
 * cannot allocate device memory: a host that owns every device buffer and forbids allocation in its
 * step callback, or code running under a fixed memory budget. The dr ping-pong buffers and the barrier words (`dr`, `dr_tmp`, `sync` of the
 * argument struct, which are ignored here) live in a file-scope device array of the library, sized
 * for m * batch <= FLYB_OPTIC_NOALLOC_MAX unit-flies (2 x 4 MiB + 256 B, held by every GPU that loads
 * the library until the process exits); larger requests return FLYB_ETOOBIG. The caller still passes
 * the state (v, adapt), the held inputs, the constants and, for a persistent launch, `status`.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress, with that
 * device current) and should come before any stream capture. Every call shares the array: calls
 * that overlap on the GPU (other streams, other threads) race on it and must be serialised; each
 * call recomputes dr from v and clears the barrier words, so no state carries over between calls.
 * The dr of the final state stays in the library's array and is not returned: a caller that needs
 * it (the whole-fly step feeds it to the W_sr drive product) computes clip(v + b, 0, 1) - b from v.
 * The looked-up address is kept per device ordinal for the life of the process; after a
 * cudaDeviceReset the library's module is loaded anew, so do not call this entry point after a
 * device reset in the same process. */
#define FLYB_OPTIC_NOALLOC_MAX (1 << 20)
int flyb_optic_run_noalloc(const flyb_optic_args* a, void* stream);

/* y[rows][batch] (+)= clamp(alpha * (M @ x'), lo, hi) with
 * x'[j][b] = clamp(x[xmap(j)][b] / x_div, x_lo, x_hi) (xmap = identity when x_index is null;
 * a correctly rounded division, as torch's `rate / 100.0` at flyverse/optic.py:572)
 * and the result row i written at y[ymap(i)]. accumulate != 0 adds into y.
 * x and y use the stated fly-minor layout with `x_rows` / `y_rows` leading rows. */
/* The optic substep's unit update after its products, for the configurations that are not the
 * fused substep: the slow receptor tone (receptor_model "full") and the per-stream hooks (the
 * substep of flyverse/optic.py:526-551). rec = gain_rr x the recurrent product (with the hooks, of
 * the rest block on dr plus each stream block on its transformed signal). classes 0: the plain
 * order, inp = ((rec + pr) - adapt_gain adapt) + spk. classes 1..FLYB_SLOW_MAX_CLASSES: per class c
 * the tone relaxes towards scale[c] x (held[c] + rec_slow[c]) with factor decay[c]; g_slow = the
 * sum over classes; inp = (rec + pr) + spk with the tone added (FLYB_SLOW_ADDITIVE), multiplying it
 * by clamp(1 + g_slow / norm, clip_lo, clip_hi) (FLYB_SLOW_GAIN), or left as is
 * (FLYB_SLOW_THRESHOLD, where the caller shifts dr by min(g_slow, 0.9 norm) before the products),
 * minus adapt_gain adapt. Then v <- inp + (v - inp) a and adapt <- dr + (adapt - dr) a_ad.
 * rec_slow[c] = gain_rr W_slow_rr[c] dr (or null), held[c] = gain_fb W_slow_rs[c] s for the frame
 * (or null). State [m][batch]. */
typedef struct flyb_optic_unit_args {
  int m;
  int batch;
  int classes;           /* 0..FLYB_SLOW_MAX_CLASSES */
  int mode;              /* with classes > 0: FLYB_SLOW_ADDITIVE, FLYB_SLOW_GAIN or FLYB_SLOW_THRESHOLD */
  float adapt_gain, a_ad, norm, clip_lo, clip_hi;
  float scale[FLYB_SLOW_MAX_CLASSES];
  float decay[FLYB_SLOW_MAX_CLASSES];
  float* v;
  float* adapt;
  float* g_slow;         /* with classes > 0 */
  float* g_cls[FLYB_SLOW_MAX_CLASSES];
  const float* held[FLYB_SLOW_MAX_CLASSES];
  const float* rec_slow[FLYB_SLOW_MAX_CLASSES];
  const float* rec;
  const float* pr;
  const float* spk;
  const float* dr;
  const float* a;        /* [m] per-unit membrane factor */
} flyb_optic_unit_args;

int flyb_optic_unit_step(const flyb_optic_unit_args* a, void* stream);

typedef struct flyb_spmm_args {
  int rows, cols, batch;
  int accumulate;
  const int* ptr; const int* col; const float* w;
  const float* x; const int* x_index; int x_rows;
  float x_div, x_lo, x_hi;
  float* y; const int* y_index; int y_rows;
  float alpha, y_lo, y_hi;
  int warps_per_row;     /* 1, 2, 4 or 8 warps share one row (0 = 1): more for long rows */
} flyb_spmm_args;

int flyb_spmm(const flyb_spmm_args* a, void* stream);

/* Optic adjoint over one checkpoint segment, run backwards from step nsteps-1 to 0.
 * Given the stored v_t and inp_t of the segment and the incoming adjoints lam_v / lam_a
 * (of v and adapt after the segment), it leaves the adjoints at the segment start in
 * lam_v / lam_a and accumulates
 *   g_edge[e] += sum_t sum_b mu[t][i][b] * dr[t][j][b]      (e = (i <- j) in W_rr CSR order)
 *   g_a[i]    += sum_t sum_b lam_v[t+1][i][b] * (v[t][i][b] - inp[t][i][b])
 * where mu = (1 - a) * lam_v. W^T is given as CSR of the transpose with `t_perm` mapping each
 * transposed entry to its CSR entry index. */
typedef struct flyb_adjoint_args {
  int m, batch, nsteps;
  int launch;
  int block, grid;
  int pad0, pad1;
  const int* t_ptr; const int* t_col; const float* t_w; const int* t_perm;  /* W_rr^T CSR */
  const float* v_hist; const float* inp_hist;        /* [nsteps][m][batch] from forward */
  const float* a; const float* b;
  float gr, ga, aad;
  int pad2;
  float* lam_v; float* lam_a;                          /* [m][batch] in/out              */
  float* lam_tmp;                                      /* [m][batch] scratch             */
  float* mu;                                           /* [m][batch] scratch             */
  float* g_edge;                                       /* [nnz] per-edge accumulator     */
  float* g_a;                                          /* [m] d/d a_i accumulator        */
  int* status; int* sync;
} flyb_adjoint_args;

int flyb_optic_adjoint(const flyb_adjoint_args* a, void* stream);

/* Segmented gather-sum in FP32 (device arrays): out[s] = alpha * sum_{seg_ptr[s] <= e < seg_ptr[s+1]}
 * x[idx[e]] * w[idx[e]] (w null: 1), summed in a fixed order (deterministic). The adjoint's
 * parameter gradients: per pair gain, the per-edge accumulator over the pair's edges times
 * gr * W0; per time constant, g_a * a over the type's units. No counterpart in the reference
 * (its gradients come from torch autograd). */
int flyb_segment_sum(const int* seg_ptr, const int* idx, const float* x, const float* w, float alpha, float* out,
                     int segments, void* stream);

/* Photoreceptor stage (flyverse/optic.py:496-517), fly-minor:
 * rad [batch][n_col][4] -> I_pr -> column x family mean -> low-pass / adaptation -> contrast,
 * writes a_pr [n_pr][batch]. `fresh` [batch] bytes are consumed (cleared). */
typedef struct flyb_photo_args {
  int n_pr, n_col, batch;
  int pad0;
  const float* rad;        /* [batch][n_col][4]                  */
  const int* pr_column;    /* [n_pr]                             */
  const float* sens;       /* [n_pr][4]                          */
  const int* avg_ptr; const int* avg_idx; const float* avg_w;  /* (n_col*5) x n_pr CSR */
  const int* pr_cell;      /* [n_pr] -> column*5 + family        */
  const unsigned char* has;/* [n_col*5]                          */
  float* I_lp; float* I_mean; float* contrast;   /* [batch][n_col*5] (reference layout) */
  unsigned char* fresh;    /* [batch]                            */
  float a_lp, c_lp;        /* low-pass coefficient exp(-dt/tau_lp) and 1 - it (rounded from double) */
  float a_ad, c_ad;        /* adaptation coefficient and 1 - it  */
  float eps, clip_hi;
  float* a_pr;             /* [n_pr][batch] output                */
} flyb_photo_args;

int flyb_photoreceptor(const flyb_photo_args* a, void* stream);

/* Motor readout on the native layout: out[b * groups + k] = mean of rates[i][b] over the members
 * i = idx[ptr[k]:ptr[k+1]] of group k, summed in member order in double (the reference's
 * launch_means, neural.cu:133-144, without the batch-major copy of the rates); rates [n][batch]. */
int flyb_group_means(const int* ptr, const int* idx, const float* rates, double* out, int groups, int batch,
                     void* stream);

/* ---------------------------------------------------------------- the eye's ray tracer
 * Replaces World.trace / BatchWorld.trace (flyverse/world.py:214, flyverse/batch_world.py:77) and the
 * column averaging of BatchSim.column_radiance (flyverse/batch_sim.py:192-201). Every scene of a
 * batch has the same primitive counts; scene b is flyb_trace_scene_floats(...) floats at
 * scene + b * that count:
 *   spheres [n_sph][6] centre xyz, radii xyz; boxes [n_box][6] lo xyz, hi xyz;
 *   planes [n_pln][6] point xyz, unit normal xyz;
 *   materials [n_sph + n_box + n_pln + 1][16] reflectance 4, second reflectance 4, emission 4,
 *     pattern period, pattern id (0 plain, 1 checks, 2 wall stripes, 3 planks), 2 unused; the last
 *     row belongs to rays that hit nothing;
 *   light [12] position xyz, colour 4, ambient 4, 1 unused.
 * Rays: explicit origins and directions ([batch][rays][3] each), or one origin per scene
 * (shared_origin) with explicit directions, or one origin per scene with body-frame directions
 * eye_dirs [rays][3] turned by pose [batch][9] (forward, left, up: d = x f + y l + z u, in double,
 * then rounded to float). With samples > 1, each run of `samples` consecutive rays is one output,
 * the weighted sum of their radiance in sample order. out is [batch][rays / samples][4], 16-byte
 * aligned. */
typedef struct flyb_trace_args {
  int batch;
  int rays;
  int n_sph;
  int n_box;
  int n_pln;
  int shared_origin;
  int samples;
  float detail;           /* surface-noise amplitude; 0 = flat colours */
  const float* scene;
  const float* origins;
  const float* dirs;
  const double* eye_dirs;
  const double* pose;
  const float* weights;   /* [samples] */
  float* out;
} flyb_trace_args;

/* floats per packed scene, or -1 for negative counts or more than 512 primitives */
int flyb_trace_scene_floats(int n_sph, int n_box, int n_pln);
int flyb_trace(const flyb_trace_args* a, void* stream);

/* Device facts for grid sizing: SM count and co-resident blocks per SM for the persistent
 * kernels at `block` threads. kind: 0 LIF, 1 optic, 2 adjoint. */
int flyb_occupancy(int kind, int block, int* sm_count, int* blocks_per_sm);

/* Failure-detection self test: one thread polls `flag` (device int, never set by anyone) through the
 * same bounded wait the grid barriers use, gives up after `spins` polls and records FLYB_EBARRIER in
 * status[0] (where = 2). Lets a host check that a wait that cannot complete ends with an error
 * status instead of a hang. No counterpart in the reference. */
int flyb_selftest_wait(const int* flag, int* status, long long spins, void* stream);

/* Measurement aid, no counterpart in the reference: gathers n_idx random rows of 64 floats
 * (x[idx[e]][0:64], x is [rows][64], 16-byte aligned) the way the optic substep gathers dr at 64
 * flies, without its arithmetic, with SMs x blocks_per_sm (1-16) blocks of 256 threads; `out`
 * takes one float per thread (SMs x blocks_per_sm x 256). Timing it gives the L2 -> SM gather rate
 * that bounds the optic kernel. Out-of-range indices are skipped. */
int flyb_gather_probe(const float* x, int rows, const int* idx, int n_idx, float* out, int blocks_per_sm,
                      void* stream);

/* Library version string. */
const char* flyb_version(void);

/* sizeof of the argument structs, in header order (lif, optic, spmm, adjoint, photo), so a
 * binding can check its mirror of this header. Returns the number of sizes written. */
int flyb_abi_sizes(int* sizes, int n);

#ifdef __cplusplus
}
#endif
#endif /* FLYB200_H */
