/*
 * relaybp.h - C ABI of the B200-native Relay-BP-S decoder (librelaybp.so).
 *
 * Plain C: opaque handles, plain pointers, sizes and int status codes.  No C++
 * exception crosses this boundary and no torch type appears in it.  Device
 * buffers passed to rbp_decode are allocated and owned by the caller (e.g. a
 * torch tensor's data pointer); the library owns only the device copies made
 * at create time (graph, priors, gamma tables) and a 4-byte work-queue counter
 * per decoder.  The stream argument is a cudaStream_t passed as void*.
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the quantum-supercomputing/pelagos tree).
 *
 * Thread safety: a decoder may be used from one host thread at a time; two
 * decoders are independent.  Error strings are kept per host thread.
 */
#ifndef RELAYBP_H_
#define RELAYBP_H_

#include <stdint.h>

#if defined(__GNUC__)
#define RBP_API __attribute__((visibility("default")))
#else
#define RBP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define RBP_OK 0
#define RBP_ERR_ARGUMENT 1     /* invalid argument; see rbp_last_error() */
#define RBP_ERR_CUDA 2         /* a CUDA runtime call failed */
#define RBP_ERR_UNSUPPORTED 3  /* problem outside this build's limits (sizes, degrees) */

/* message storage types; posteriors and memory accumulate in f32 (f64 for F64) */
#define RBP_MSG_F32 0
#define RBP_MSG_F16 1
#define RBP_MSG_BF16 2
#define RBP_MSG_F64 3

/* rounding of the memory mix  (1 - g) * llr + g * posterior */
#define RBP_MIX_SEPARATE 0     /* every product and sum rounded once */
#define RBP_MIX_FMA_GP 1       /* fma(g, posterior, (1 - g) * llr) */
#define RBP_MIX_FMA_LP 2       /* fma(1 - g, llr, g * posterior) */

typedef struct rbp_graph rbp_graph;
typedef struct rbp_decoder rbp_decoder;

/* Last error message of the calling host thread ("" when none). */
RBP_API const char* rbp_last_error(void);

/* Library version string. */
RBP_API const char* rbp_version(void);

/*
 * Tanner graph in the reference's edge-centric form, copied to `device`.
 * Replaces CSRGraph(H_csr, device) and _build_edge_representation
 * (src/pelagos/graph.py:31-211): edge e is the e-th nonzero of the CSR matrix,
 * chk_ptr[C+1] delimits each check's edges, edge_var[E] is the variable of
 * each edge, and var_edges[var_ptr[v]..var_ptr[v+1]) lists variable v's edges
 * in the order their check messages are summed (graph.py:145 argsort order).
 * All arrays are host memory.
 */
RBP_API int rbp_graph_create(int32_t C, int32_t V, int32_t E,
                     const int32_t* chk_ptr, const int32_t* edge_var,
                     const int32_t* var_ptr, const int32_t* var_edges,
                     int32_t device, rbp_graph** out);
RBP_API int rbp_graph_destroy(rbp_graph* g);

/* Decode parameters: the RelayBPDecoder constructor arguments that reach the
 * decode loop (src/pelagos/decoder.py:271-307). */
typedef struct {
  int32_t pre_iter;         /* first-phase iterations (ordered memory) */
  int32_t num_sets;         /* relay legs */
  int32_t set_max_iter;     /* iterations per relay leg */
  int32_t stop_nconv;       /* solutions a shot collects before it stops */
  int32_t msg_type;         /* RBP_MSG_* */
  int32_t last_leg;         /* 1: unconverged shots return the final hard decision */
  int32_t use_alpha;        /* normalized min-sum with per-iteration alpha table */
  int32_t use_beta;         /* offset min-sum */
  float beta;
  int32_t mix_mode;         /* RBP_MIX_* */
} rbp_params;

/*
 * Decoder: graph + parameters + device copies of the prior LLRs [V], the
 * leg memory-strength table [num_sets, V] (row l = relay leg l) and the
 * per-iteration alpha table [n_alpha].  Replaces RelayBPDecoder.__init__
 * (src/pelagos/decoder.py:271-784) from the graph build onward; the gamma
 * table stands for the per-leg draws of decoder.py:3684-3700.
 * llr, gamma_legs and alpha are host memory; gamma_legs may be NULL when
 * num_sets == 0 and alpha may be NULL when use_alpha == 0.
 */
RBP_API int rbp_decoder_create(const rbp_graph* g, const rbp_params* p,
                       const float* llr, const float* gamma_legs,
                       const float* alpha, int32_t n_alpha, rbp_decoder** out);
RBP_API int rbp_decoder_destroy(rbp_decoder* d);

/* Replace the shared prior LLRs (and the selection weights derived from
 * them) for later decodes; host memory [V].  Replaces
 * RelayBPDecoder.override_llr_columns (src/pelagos/decoder.py:785-834). */
RBP_API int rbp_decoder_set_llr(rbp_decoder* d, const float* llr);

/* Launch shape (no reference counterpart: the reference autotunes Triton
 * tile sizes instead, src/pelagos/autotune.py:302-541).  A group of
 * `group_threads` threads (a multiple of 32, at most 1024) decodes
 * `shots_per_group` shots at once (1 or 2) and a thread block holds
 * `groups_per_block` such groups.  groups_per_block 1, or two shots per
 * group, selects the block-per-group kernel (check degrees up to 16); 0 (or
 * -1) the kernel whose blocks hold as many one-shot groups as fit.  Zeros pick
 * the defaults.  Results do not depend on the shape.  Fails with
 * RBP_ERR_UNSUPPORTED when the shape's registers or shared memory do not fit.
 * Sets the shape of every launch kind (rbp_decoder_configure_kind with
 * RBP_LAUNCH_ALL and one resident block per SM). */
RBP_API int rbp_decoder_configure(rbp_decoder* d, int32_t group_threads, int32_t groups_per_block,
                                  int32_t shots_per_group);

/* Launch kinds.  A decode launch whose rbp_batch.skip_relay_legs is set runs
 * the pre-iterations only, so no shot runs more than pre_iter iterations in
 * it; such launches use the RBP_LAUNCH_PRE shape, every other launch the
 * RBP_LAUNCH_LEGS shape. */
#define RBP_LAUNCH_ALL 0
#define RBP_LAUNCH_PRE 1
#define RBP_LAUNCH_LEGS 2

/* Launch shape of one launch kind (no reference counterpart, like
 * rbp_decoder_configure).  blocks_per_sm 2 selects the block-per-group kernel
 * compiled for two resident blocks per SM (groups_per_block 1 and
 * shots_per_group 1 only; half the register file per block, so
 * group_threads is at most 512 for up to 4 owned variables per thread, 448
 * for 6, 384 for 8 and 256 for 12 or 16): two shots decode side by side on an
 * SM, each at a longer iteration latency, which raises throughput and can
 * lengthen a batch whose slowest shot bounds it.  0 or 1: the kernels compiled
 * for one resident block.  Results do not depend on the shape. */
RBP_API int rbp_decoder_configure_kind(rbp_decoder* d, int32_t kind, int32_t group_threads,
                                       int32_t groups_per_block, int32_t shots_per_group,
                                       int32_t blocks_per_sm);

/* Shared-memory bytes of one shot's region and of the block-wide tables for
 * the current message type; the RBP_LAUNCH_LEGS shape currently configured.
 * Any pointer may be NULL. */
RBP_API int rbp_decoder_query(const rbp_decoder* d, int64_t* group_smem, int64_t* block_smem,
                      int32_t* group_threads, int32_t* groups_per_block, int32_t* blocks,
                      int32_t* shots_per_group);

/* The shape configured for launch kind RBP_LAUNCH_PRE or RBP_LAUNCH_LEGS;
 * blocks_per_sm is the resident-block count the kernel is compiled for and
 * blocks the persistent grid.  Any pointer may be NULL. */
RBP_API int rbp_decoder_query_kind(const rbp_decoder* d, int32_t kind, int32_t* group_threads,
                                   int32_t* groups_per_block, int32_t* shots_per_group,
                                   int32_t* blocks_per_sm, int32_t* blocks);

/* Per-call inputs (device memory).  Optional pointers may be NULL.
 * Mirrors decode()'s keyword arguments (src/pelagos/decoder.py:2317-2361).
 * struct_size must hold sizeof(rbp_batch) (RBP_BATCH_SIZE): a caller whose
 * declaration of the struct has other fields (an older or hand-written
 * binding) is rejected with RBP_ERR_ARGUMENT before any field is read. */
typedef struct {
  uint32_t struct_size;            /* sizeof(rbp_batch) */
  const uint8_t* syndromes;        /* [B, C] bits in the low bit of each byte */
  const float* llr_per_shot;       /* [B, V] prior_llr, overrides the shared LLRs */
  const float* gamma_pre;          /* [B, V] init_gamma for the first phase */
  float gamma0;                    /* first-phase strength when gamma_pre is NULL (0 for algo=plain) */
  const float* init_posterior;     /* [B, V] posterior the first phase starts from */
  const float* gamma_legs_shot;    /* [B, shot_leg_rows, V] per-shot strengths of legs < n_shot_legs */
  int32_t n_shot_legs;
  int32_t pre_iter;                /* first-phase iterations for this call (pre_iter_override) */
  int32_t skip_relay_legs;         /* 1: stop after the first phase */
  /* Resumable decoding (rbp_state_bytes bytes per shot, device memory).  With
   * resume_state, each shot continues from its saved state at relay leg
   * legs_begin instead of starting with the pre-iterations; relay legs run up to
   * (excluding) legs_end (<= 0: all).  With suspend_state, each shot's state
   * after the last phase run is saved.  The two may be the same buffer; both
   * must be 16-byte aligned.  No reference counterpart: the reference's
   * fast_max_unconverged_pct exit (decoder.py:2890-2935) is built on it. */
  const void* resume_state;
  void* suspend_state;
  int32_t legs_begin;
  int32_t legs_end;
  /* Rows per shot in gamma_legs_shot (0: n_shot_legs).  Leg l < n_shot_legs
   * uses row min(l, shot_leg_rows - 1), so one row can serve several legs. */
  int32_t shot_leg_rows;
  /* Order in which the persistent kernel takes the shots (device [B], a
   * permutation of 0..B-1), or NULL for 0, 1, ..., B-1.  Results do not depend
   * on it; putting the shots that will run longest first keeps them from
   * finishing after everything else.  Entries outside [0, B) are skipped. */
  const int32_t* shot_order;
  /* Device int32: only queue positions below it are taken (NULL: all B). */
  const int32_t* queue_len;
  /* Split decode.  After the pre-iterations (or when resumed at leg 0 with a
   * solution found), a shot that found a solution runs
   * relay legs l < solved_legs with the constant strength solved_gamma; with
   * suspend_unsolved = 1 (which needs suspend_state) a shot that found none
   * saves its state there and stops, to be resumed by a later call, and only
   * such shots write their state. */
  float solved_gamma;
  int32_t solved_legs;
  int32_t suspend_unsolved;
  /* When to test an iteration's parity before its min-sum pass, skipping that
   * pass when every check holds: 0 never (one fused pass), 1 at the first
   * testable iteration of each relay leg, 2 at every iteration.  Results do
   * not depend on it; it pays off where legs converge at once. */
  int32_t parity_first;
} rbp_batch;

/* Outputs (device memory).  Any may be NULL except found_count/iterations.
 * struct_size must hold sizeof(rbp_outputs) (RBP_OUTPUTS_SIZE), as for rbp_batch. */
typedef struct {
  uint32_t struct_size;            /* sizeof(rbp_outputs) */
  uint8_t* errors;                 /* [B, V] 0/1 */
  uint32_t* errors_packed;         /* [B, ceil(V/32)] bit v%32 of word v/32 */
  float* weights;                  /* [B] selected solution weight, +inf when none */
  int64_t* weight_fixed;           /* [B] exact weight in units of 2^-32, INT64_MAX when none */
  int32_t* found_count;            /* [B] solutions found */
  int32_t* iterations;             /* [B] BP iterations the shot ran */
  void* last_posterior;            /* [B, V] f32 (f64 for RBP_MSG_F64) posterior at the end */
} rbp_outputs;

#define RBP_BATCH_SIZE ((uint32_t)sizeof(rbp_batch))
#define RBP_OUTPUTS_SIZE ((uint32_t)sizeof(rbp_outputs))

/* Bytes of one shot's saved state (rbp_batch.resume_state / suspend_state). */
RBP_API int rbp_state_bytes(const rbp_decoder* d, int64_t* bytes_per_shot);

/* Byte offset of the posterior ([V] f32, f64 for RBP_MSG_F64) inside a saved state. */
RBP_API int rbp_state_posterior_offset(const rbp_decoder* d, int64_t* offset);

/*
 * Decode B shots on `stream`.  Asynchronous: returns after the launch.
 * Replaces RelayBPDecoder.decode (src/pelagos/decoder.py:2317-2449) and its
 * single-GPU loop _decode_loop_single_gpu (decoder.py:3394-3873) with all its
 * per-iteration kernels (src/pelagos/kernels.py:609-1350).
 */
RBP_API int rbp_decode(rbp_decoder* d, int64_t B, const rbp_batch* in, const rbp_outputs* out,
               void* stream);

/*
 * Mixed-code launch: several decoders' batches in ONE persistent launch.
 * Each thread block serves one code at a time, with that code's group shape,
 * and takes shots from that code's work queue; when the queue is empty the
 * block moves to the next code that still has shots.  Shots of small and large
 * codes therefore share the GPU without a launch per code, and converged shots
 * free their group for any code's remaining work.  Extends the reference's
 * per-decoder, per-batch-size decode (src/pelagos/decoder.py:1480-1538) and the
 * host-side "difficult batch" re-queue of pelagos_benchmark.py:1462-1520.
 * Up to 8 decoders, all on one device, float32 messages.
 */
typedef struct rbp_mixed rbp_mixed;

RBP_API int rbp_mixed_create(const rbp_decoder* const* decoders, int32_t n, rbp_mixed** out);
RBP_API int rbp_mixed_destroy(rbp_mixed* m);

/* Decode batch i (B[i] shots, ins[i], outs[i]) with decoders[i], for all i,
 * in one launch on `stream` (asynchronous). */
RBP_API int rbp_mixed_decode(rbp_mixed* m, const int64_t* B, const rbp_batch* ins, const rbp_outputs* outs,
                             void* stream);

/* Record the same decode (same sizes and buffers) as a CUDA graph (the queue
 * reset and the persistent launch); rbp_mixed_replay launches that graph on
 * `stream`.  A replay reads the captured input buffers and writes the captured
 * output buffers, so callers refill the inputs in place between replays. */
RBP_API int rbp_mixed_capture(rbp_mixed* m, const int64_t* B, const rbp_batch* ins, const rbp_outputs* outs);
RBP_API int rbp_mixed_replay(rbp_mixed* m, void* stream);

/* Launch shape of code i inside the mixed launch. */
RBP_API int rbp_mixed_query(const rbp_mixed* m, int32_t i, int32_t* group_threads, int32_t* groups_per_block,
                            int32_t* block_threads, int32_t* blocks);

/* Set each code's group size inside the mixed launch (group_threads[i]; 0 keeps
 * code i's current size): a multiple of 32 that divides the launch's block size
 * and leaves each thread at most the instantiation's variables and 32 checks.
 * Each code gets as many groups per block as fit.  Drops a captured graph.
 * The autotuner's hook; no reference counterpart. */
RBP_API int rbp_mixed_configure(rbp_mixed* m, const int32_t* group_threads);

/* Size of the scratch array that rbp_decode_static uses (1 MiB per GPU). */
#define RBP_STATIC_SCRATCH_BYTES (1 << 20)

/*
 * Decode B shots without allocating anything.  This entry point has no
 * counterpart in the reference.
 *
 * It is for callers that cannot call cudaMalloc while they decode: a real-time
 * decoding service with a fixed device-memory budget, which cannot afford the
 * device-wide synchronisation and unbounded latency of an allocation between
 * syndrome rounds, or a process whose device memory is already reserved by
 * another allocator (for example torch's caching allocator), where a new
 * allocation may fail.
 *
 * It takes the whole problem in one call, with no rbp_graph or rbp_decoder:
 *   - the graph as host arrays, exactly as for rbp_graph_create;
 *   - the parameters;
 *   - device pointers to the prior LLRs [V], the leg table [num_sets, V] and
 *     the alpha table [n_alpha] (may be NULL when use_alpha == 0);
 *   - the batch inputs and outputs, as for rbp_decode.
 * It decodes with the same kernel as rbp_decode, so the results are identical.
 *
 * The graph tables it derives (check degrees, check pointers, slot positions)
 * and the kernel's work-queue counter live in a static device array of
 * RBP_STATIC_SCRATCH_BYTES bytes.  That array is part of the library image:
 * every GPU that loads the library holds it until the process exits.  A graph
 * whose tables need more returns RBP_ERR_UNSUPPORTED.  The call neither
 * allocates nor frees memory, on the device or on the host; it stages the
 * tables through a fixed stack buffer.
 *
 * All calls share that one array, and each call overwrites it: the counter is
 * cleared and every table is rewritten.  Calls that overlap on the GPU (on
 * different streams, or from different host threads) therefore race and give
 * wrong results; serialise them on one stream.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and caches it; host threads may make that first call
 * concurrently.  Make that first call before any stream capture begins.
 *
 * The tables are copied from host memory that exists only during the call, so
 * a call on a stream that is being captured returns RBP_ERR_UNSUPPORTED
 * without enqueuing anything: a recorded copy would read freed memory when
 * the graph is replayed.  The graph arrays are checked as rbp_graph_create
 * checks them (RBP_ERR_ARGUMENT for a var_edges that is not the
 * variable-major permutation of edge_var).
 */
RBP_API int rbp_decode_static(int32_t C, int32_t V, int32_t E,
                              const int32_t* chk_ptr, const int32_t* edge_var,
                              const int32_t* var_ptr, const int32_t* var_edges,
                              const rbp_params* p, const float* llr, const float* gamma_legs,
                              const float* alpha, int32_t n_alpha, int32_t device,
                              int64_t B, const rbp_batch* in, const rbp_outputs* out, void* stream);

/*
 * Learned relay-leg proposal (no counterpart in the reference).
 *
 * A 2-layer edge-conditioned message-passing network on the Tanner graph
 * (node width 64, message width 16, bf16 weights, fp32 sums) that reads a
 * shot's syndrome and its posterior after the pre-iterations and proposes
 * per-variable memory strengths for the first relay legs.  The strengths are
 * handed to rbp_decode as rbp_batch.gamma_legs_shot, the per-shot form of the
 * reference's explicit_gammas rows (src/pelagos/decoder.py:338-340, 481-491,
 * 3685-3688), inside gamma_dist_interval (src/pelagos/utils.py:128-160).
 * Every decoded error still has to satisfy H e = s and is still ranked by the
 * decoder's weight rule; later legs keep the seeded table.
 *
 * The network owns its parameters (fp32 master copy, bf16 working copy, AdamW
 * moments) and a training workspace sized for the largest batch seen.
 */
typedef struct rbp_net rbp_net;

typedef struct {
  float lr;            /* AdamW step size; 0 computes the loss and gradients only */
  float beta1, beta2, eps, weight_decay;
  float w_neg;         /* loss weight of variables whose pre-iteration decision is wrong */
} rbp_net_hparams;

/* Number of network parameters (the length of the flat parameter vector). */
RBP_API int rbp_net_param_count(int64_t* n);

/* Network on graph g's device; llr is the host [V] prior LLR vector.  Parameters start at 0. */
RBP_API int rbp_net_create(const rbp_graph* g, const float* llr, rbp_net** out);
RBP_API int rbp_net_destroy(rbp_net* n);

/* Copy the flat fp32 parameters in (device pointer; resets the AdamW state) or out. */
RBP_API int rbp_net_set_params(rbp_net* n, const float* theta, void* stream);
RBP_API int rbp_net_get_params(const rbp_net* n, float* theta, void* stream);

/* Training-path forward: logits r [B, V] (device).  syn [B, C] uint8, post [B, V] f32. */
RBP_API int rbp_net_forward(rbp_net* n, int64_t B, const uint8_t* syn, const float* post, float* logits,
                            void* stream);

/* One training step on B shots: forward, the weighted logistic loss against
 * target [B, V] (1 where the pre-iteration hard decision equals the true error),
 * backward, and (lr > 0) an AdamW update.  loss (device [1]) and grads (device
 * [n]) receive the loss and the gradient when not NULL. */
RBP_API int rbp_net_train_step(rbp_net* n, int64_t B, const uint8_t* syn, const float* post, const uint8_t* target,
                               const rbp_net_hparams* hp, float* loss, float* grads, void* stream);

/* Inference on the tensor cores: gammas [B, V] = lo + (hi - lo) sigmoid(r) and/or
 * logits [B, V].  Shot b's posterior is post[b * post_stride ...] (post_stride
 * 0: V), so it can be read straight out of saved decode states
 * (rbp_state_posterior_offset).  With shot_list (device [B]) only the shots shot_list[i],
 * i < *list_count (a device int32; all B entries when list_count is NULL),
 * are evaluated and their rows written; other rows are left as they are, so a
 * caller can evaluate a subset chosen on the device without a host round trip.
 * Needs a graph below 65536 edges whose per-shot state fits in one block's
 * shared memory (RBP_ERR_UNSUPPORTED otherwise). */
RBP_API int rbp_net_propose(rbp_net* n, int64_t B, const uint8_t* syn, const float* post, int64_t post_stride,
                            float lo, float hi, const int32_t* shot_list, const int32_t* list_count, float* gammas,
                            float* logits, void* stream);

/*
 * GF(2) product of a sparse 0/1 matrix (device CSR: row_ptr [R+1], cols) with
 * each of B rows of x (device uint8 [B, N], only bit 0 read): out[b, r] =
 * XOR_{j in row r} x[b, j] (device uint8 [B, R]).  Replaces the host-side
 * products of the reference's observable runner, s = H e and O e
 * (src/pelagos/adapter.py:545-560, 601-613, 679).  N <= 49,152.
 */
RBP_API int rbp_gf2_matvec(const uint8_t* x, int64_t B, int32_t N, const int32_t* row_ptr, const int32_t* cols,
                           int32_t R, uint8_t* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RELAYBP_H_ */
