/*
 * hptt_cuda.h -- C ABI of libhptt_cuda.so, the B200 (sm_100a) engine for
 *
 *     B[perm(i)] = alpha * A[i] + beta * B[perm(i)]
 *
 * Column-major tensors (dimension 0 has stride 1), output extents
 * out_size[k] = in_size[perm[k]], element types float, double, complex float
 * and complex double, ranks 2..8.  All data pointers are DEVICE pointers.
 *
 * Every entry point returns an int status (HPTT_OK = 0).  No entry point
 * throws, and none takes a C++ or torch type.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * the reference project).
 */
#ifndef HPTT_CUDA_H_
#define HPTT_CUDA_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Element types.  Reference: hptt::FloatComplex / DoubleComplex
 * (inc/hptt/types.h:21-22) and the four explicit instantiations
 * (inc/hptt/hptt.h:99-123). */
enum hptt_cuda_dtype {
  HPTT_CUDA_F32 = 0,
  HPTT_CUDA_F64 = 1,
  HPTT_CUDA_C64 = 2,  /* float _Complex, layout of float2  */
  HPTT_CUDA_C128 = 3  /* double _Complex, layout of double2 */
};

/* Status codes.  The reference returns nullptr from create_plan for the
 * argument errors 1-5 (inc/hptt/hptt.h:71-83, src/hptt.cc:25-56); here each
 * cause has its own code. */
enum hptt_cuda_status {
  HPTT_OK = 0,
  HPTT_ERR_NULL_DATA = 1,
  HPTT_ERR_RANK = 2,
  HPTT_ERR_SIZE_VECTOR = 3,
  HPTT_ERR_SIZE_VALUE = 4,
  HPTT_ERR_PERM = 5,
  HPTT_ERR_DTYPE = 6,
  HPTT_ERR_CUDA = 7,
  HPTT_ERR_NO_DEVICE = 8,
  HPTT_ERR_ALLOC = 9,
  HPTT_ERR_BUDGET = 10,
  HPTT_ERR_HANDLE = 11,
  HPTT_ERR_TIMEOUT = 12,
  HPTT_ERR_TOO_LARGE = 13,
  HPTT_ERR_BUSY = 14,
  HPTT_ERR_LABELS = 15,
  HPTT_ERR_BLAS = 16
};

typedef struct hptt_cuda_plan_s *hptt_cuda_plan_t;

/*
 * Create a transpose plan.
 * Replaces: hptt::create_plan<T> (inc/hptt/hptt.h:85-93, src/hptt.cc:16-93)
 * and the per-type factories create_trans_plan_impl_{s,d,c,z}
 * (inc/hptt/impl/hptt_trans_impl.h:81-103, src/impl/hptt_trans_impl_s.cc:8-20).
 *
 *   in_size[rank], perm[rank]   as in the reference; rank >= 2
 *   in_outer / out_outer        outer (padded) sizes or NULL; out_outer is
 *                               indexed by OUTPUT dimension
 *                               (inc/hptt/hptt.h:58-61)
 *   alpha, beta                 two doubles each (re, im).  With
 *                               complex_scalars == 0 only [0] is used, as a
 *                               real scalar (the reference's
 *                               DeducedFloatType, inc/hptt/types.h:29-54);
 *                               complex_scalars != 0 (complex types only)
 *                               applies full complex scalars -- an
 *                               extension the reference cannot express.
 *   in, out                     device pointers; never freed by the plan
 *   num_threads                 accepted and ignored (GPU launch shape is
 *                               chosen by the planner)
 *   tuning_timeout              0: heuristic only; != 0: time candidate tile
 *                               shapes on scratch buffers (< 0 all of them,
 *                               > 0 for at most that many seconds) and cache
 *                               the winner (inc/hptt/hptt.h:48-57)
 * B is read only when |beta| >= 1e-16 (inc/hptt/impl/hptt_trans_impl.h:75-78).
 */
int hptt_cuda_plan_create(int dtype, uint32_t rank, const uint32_t *in_size,
                          const uint32_t *perm, const uint32_t *in_outer,
                          const uint32_t *out_outer, const double *alpha,
                          const double *beta, int complex_scalars,
                          const void *in, void *out, uint32_t num_threads,
                          double tuning_timeout, hptt_cuda_plan_t *plan);

/* Enqueue the transpose on the plan's stream (asynchronous).
 * Replaces: CGraphTransPackBase::exec() / operator()()
 * (inc/hptt/impl/hptt_trans.h:26-27). */
int hptt_cuda_plan_exec(hptt_cuda_plan_t plan);

/* Same, on an explicit cudaStream_t (passed as void*). Extension. */
int hptt_cuda_plan_exec_on(hptt_cuda_plan_t plan, void *stream);

/* Swap the data pointers; sizes, perm, scalars and tile choice are kept.
 * Replaces: CGraphTransPackBase::reset_data (inc/hptt/impl/hptt_trans.h:29,
 * inc/hptt/cgraph/cgraph_trans.tcc:64-68).  Like the reference it does not
 * re-validate; a null pointer is rejected at exec instead. */
int hptt_cuda_plan_reset_data(hptt_cuda_plan_t plan, const void *in, void *out);

/* Write a readable plan summary (NUL-terminated, truncated to len).
 * Replaces: CGraphTransPackBase::print_plan (inc/hptt/impl/hptt_trans.h:28). */
int hptt_cuda_plan_describe(hptt_cuda_plan_t plan, char *buf, size_t len);

/* Accepted no-ops: there is no host thread team on the GPU path.
 * Replaces: set_thread_ids / unset_thread_ids
 * (inc/hptt/impl/hptt_trans.h:30-31, inc/hptt/cgraph/cgraph_trans.tcc:71-83). */
int hptt_cuda_plan_set_thread_ids(hptt_cuda_plan_t plan, const int32_t *ids,
                                  uint32_t count);
int hptt_cuda_plan_unset_thread_ids(hptt_cuda_plan_t plan);

/* Stream used by hptt_cuda_plan_exec (cudaStream_t as void*; NULL = the
 * legacy default stream, the initial setting).  Extension. */
int hptt_cuda_plan_set_stream(hptt_cuda_plan_t plan, void *stream);

/* Wait for the plan's stream.  Extension (exec is asynchronous). */
int hptt_cuda_plan_sync(hptt_cuda_plan_t plan);

/* Scalars: change alpha/beta on an existing plan (re-decides whether B is
 * read).  Reference: ParamTrans::set_coef
 * (inc/hptt/param/parameter_trans.tcc:161-168), used by its tuner. */
int hptt_cuda_plan_set_coef(hptt_cuda_plan_t plan, const double *alpha,
                            const double *beta, int complex_scalars);

/* Algorithmic bytes one exec moves: 2*N*sizeof(T), plus N*sizeof(T) when B
 * is read.  Extension, for throughput reporting. */
int hptt_cuda_plan_bytes(hptt_cuda_plan_t plan, uint64_t *bytes);

/* Kernel launches one exec issues (1, or 0 for an empty problem). */
int hptt_cuda_plan_launches(hptt_cuda_plan_t plan, uint32_t *launches);

/* Destroy the plan (does not touch the user's buffers).
 * Replaces: the shared_ptr deleter of the reference plan
 * (inc/hptt/impl/hptt_trans.h:22, src/hptt.cc:86-92). */
int hptt_cuda_plan_destroy(hptt_cuda_plan_t plan);

/* Host-only dry run of create: argument guard, index fusion and tile choice,
 * without a device or data pointers.  Writes the plan summary that
 * hptt_cuda_plan_describe would print (minus the grid line).  Extension, for
 * tests and tooling.  Reference counterpart: the same guard
 * (src/hptt.cc:25-56) and ParamTrans::merge_idx_
 * (inc/hptt/param/parameter_trans.tcc:223-283). */
int hptt_cuda_plan_inspect(int dtype, uint32_t rank, const uint32_t *in_size,
                           const uint32_t *perm, const uint32_t *in_outer,
                           const uint32_t *out_outer, char *buf, size_t len);

/* Host-only replay of a launch's addressing: plans the problem, then walks
 * every tile and thread with the kernels' own index helpers and checks that
 * every access stays inside the buffers and shared memory, and that every
 * inner element of B is written exactly once with the element of A the
 * permutation maps to it.  max_vec_bytes limits vector accesses (0 = widest).
 * Where the problem allows them, it then replays vector-tile forms the tuner
 * tries (bases on and off a 16-byte boundary) and TMA-tile forms (both
 * tensor maps checked against TMA's stride, box and coordinate rules, every
 * box clipped at the tensor's edges).  Returns 0 when all checks hold, else
 * a diagnostic code >= 1000.  Extension, for tests; no reference
 * counterpart. */
int hptt_cuda_debug_check_indexing(int dtype, uint32_t rank, const uint32_t *in_size,
                                   const uint32_t *perm, const uint32_t *in_outer,
                                   const uint32_t *out_outer, int max_vec_bytes,
                                   uint64_t *checked);

/* The same replay for one vector-tile form: threads per CTA `nt`, window
 * slots per row `nvx` and per column `nvy` (8, 16 or 32), 16-byte vectors per
 * thread and phase `vj` (4 or 8), grid order `grid_order`, whether B is read
 * (`update`), and the A and B base addresses
 * `mis_a` / `mis_b` elements past a 16-byte boundary.  Returns 0 when the
 * checks hold (also when the problem takes no vector tile: *checked is then
 * 0), else a diagnostic code >= 2000.  Extension, for tests; no reference
 * counterpart. */
int hptt_cuda_debug_check_vtile(int dtype, uint32_t rank, const uint32_t *in_size,
                                const uint32_t *perm, const uint32_t *in_outer,
                                const uint32_t *out_outer, int nt, int nvx, int nvy,
                                int vj, int grid_order, int update, int mis_a, int mis_b,
                                uint64_t *checked);

/* CTAs of TMA-tile launches (KIND_TTILE) whose bounded wait for their box
 * loads ran out since the library was loaded on the current device; such a
 * CTA stores nothing.  0 in every correct run.  Extension, for tests; no
 * reference counterpart. */
int hptt_cuda_debug_tma_timeouts(uint32_t *count);

/* Size of the fixed device array hptt_cuda_transpose_noalloc keeps its
 * offset tables in (one array per GPU, held until the process exits). */
#define HPTT_NOALLOC_TABLE_BYTES 65536

/*
 * One transpose that allocates no device memory.
 *
 * No counterpart in the reference.  hptt_cuda_plan_create keeps a plan's
 * offset tables (a few KB) in device memory it obtains with cudaMalloc.
 * Callers that cannot allocate device memory when they transpose --
 * frameworks whose device memory comes only from their own pool or arena
 * (an allocation behind the pool's back breaks its accounting or fails under
 * its reservation), jobs held to a fixed device-memory budget -- use this
 * call instead.  It plans the transpose on the host (with the autotune
 * cache's entry for the problem when there is one), copies the tables into
 * a fixed HPTT_NOALLOC_TABLE_BYTES array compiled into the library, and
 * enqueues the same kernel on `stream` (cudaStream_t as void*, NULL = the
 * legacy default stream).  It never calls cudaMalloc, cudaFree or another
 * device allocator.  The table copy is a cudaMemcpyAsync from pageable host
 * memory that the call owns and frees before it returns.
 *
 * Arguments mean what they mean for hptt_cuda_plan_create; in/out are device
 * pointers the caller owns.  Returns HPTT_ERR_TOO_LARGE, before any copy or
 * launch, when this problem's tables would not fit the array.
 *
 * The array is shared by every call in the process on that GPU and keeps
 * the last call's tables: calls that can run at the same time on the GPU
 * (different streams, several host threads) race on it and must be
 * serialised by the caller; calls on one stream are ordered.  Each call
 * looks the array's address up in the current context.
 */
int hptt_cuda_transpose_noalloc(int dtype, uint32_t rank, const uint32_t *in_size,
                                const uint32_t *perm, const uint32_t *in_outer,
                                const uint32_t *out_outer, const double *alpha,
                                const double *beta, int complex_scalars, const void *in,
                                void *out, void *stream);

/* HPTT_NOALLOC_TABLE_BYTES as compiled into the library.  No counterpart in
 * the reference. */
size_t hptt_cuda_noalloc_table_bytes(void);

/*
 * Batched form: many plans in one graph launch.  No reference counterpart:
 * the reference runs each plan's exec on its own
 * (inc/hptt/cgraph/cgraph_trans.tcc:27-48); a batch replaces a loop of those
 * calls.
 *
 * A batch snapshots each plan's launch arguments (problem, tuned tile,
 * offset tables, data pointers, scalars) into a device descriptor table and
 * splits every plan's tiles into work items, grouped by tile body (element
 * storage, arithmetic, B read, tile shape).  One persistent kernel per group
 * takes its items from an atomic counter; a CUDA graph built at create holds
 * the counter reset and every group kernel as independent nodes, so the
 * groups run side by side and one graph launch runs the batch.  Results are
 * bit-identical to each plan's own exec.  The plans must outlive the batch
 * (their offset tables are shared, not copied), and no plan's output may
 * overlap another plan's input or output (entries run concurrently, in no
 * fixed order).
 *   create    build descriptors, work list and graph (synchronous uploads)
 *   refresh   re-read every plan's pointers and scalars after reset_data /
 *             set_coef on it; rebuilds the graph only if the launch shape
 *             changed
 *   exec      enqueue one run on a stream (cudaStream_t as void*; NULL =
 *             legacy default stream)
 *   info      algorithmic bytes of one exec, work items, kernels per exec
 */
typedef struct hptt_cuda_batch_s *hptt_cuda_batch_t;
int hptt_cuda_batch_create(const hptt_cuda_plan_t *plans, uint32_t count,
                           hptt_cuda_batch_t *batch);
int hptt_cuda_batch_refresh(hptt_cuda_batch_t batch);
int hptt_cuda_batch_exec(hptt_cuda_batch_t batch, void *stream);
int hptt_cuda_batch_info(hptt_cuda_batch_t batch, uint64_t *bytes, uint32_t *work_items,
                         uint32_t *kernels);
int hptt_cuda_batch_destroy(hptt_cuda_batch_t batch);

/* The per-call form a batch is compared with: exactly one
 * hptt_cuda_plan_exec_on(plans[i], stream) per plan, in order, from one C
 * loop (no interpreter between calls).  Reference counterpart: a caller's
 * loop of plan->exec() (inc/hptt/impl/hptt_trans.h:26). */
int hptt_cuda_plan_exec_many(const hptt_cuda_plan_t *plans, uint32_t count, void *stream);

/*
 * Served form: a request loop with continuous batching.  No reference
 * counterpart (the reference is a library of synchronous plans).
 *
 * A request names a plan -- its tuned tile and offset tables stay resident --
 * and optionally other device buffers of the plan's shape (in/out both NULL:
 * the plan's own).  A scheduler thread admits queued requests in arrival
 * order while the device bytes (A and B footprints) of admitted, unfinished
 * requests stay within budget_bytes; a request whose output buffer an
 * earlier unfinished request still writes waits without holding up later
 * ones.  Batched mode packs each pass's admissions (at most max_batch) into
 * one launch of the batched form's group kernels on a free stream of a pool
 * of max_inflight_launches streams, so arrivals during earlier launches run
 * in new launches that overlap them.  per_call != 0 is the baseline: one
 * plain exec per request, in arrival order, on one stream, with up to
 * max_inflight_launches requests enqueued at once.  Completions are found by
 * polling events; a request's latency is completion minus submission on the
 * host's steady clock.  Each result equals the request's own plain exec.
 *   submit      queue a request (non-blocking); *ticket identifies it.
 *               HPTT_ERR_BUDGET if it alone exceeds the budget.
 *   wait        until that request finished (its status) or timeout
 *               (HPTT_ERR_TIMEOUT)
 *   drain       until every submitted request finished
 *   stats       counters and latency percentiles since the last reset
 *   reset_stats only when nothing is outstanding (else HPTT_ERR_BUSY)
 *   run_poisson open-loop load: arrivals with exponential gaps at `rate`
 *               per second for `seconds`, each a uniformly drawn plan of
 *               `pool` on its own buffers; then drain; fills *stats
 *   destroy     finishes everything queued, then frees the server
 */
typedef struct hptt_cuda_server_s *hptt_cuda_server_t;
typedef struct {
  uint64_t budget_bytes;
  uint32_t max_inflight_launches;
  uint32_t max_batch;
  int32_t per_call;
  int32_t reserved;
} hptt_cuda_serve_config;
typedef struct {
  uint64_t submitted, completed, failed, launches, bytes;
  uint64_t peak_inflight_bytes, peak_pending;
  double elapsed_s, throughput_rps, gbs, mean_batch;
  double lat_mean_us, lat_p50_us, lat_p99_us, lat_p999_us, lat_max_us;
  double sched_pass_max_us;  /* longest pass of the scheduler thread's loop
                                (idle waits excluded): a long one means the
                                thread was held up */
} hptt_cuda_serve_stats;
int hptt_cuda_server_create(const hptt_cuda_serve_config *cfg, hptt_cuda_server_t *server);
int hptt_cuda_server_submit(hptt_cuda_server_t server, hptt_cuda_plan_t plan, const void *in,
                            void *out, uint64_t *ticket);
int hptt_cuda_server_wait(hptt_cuda_server_t server, uint64_t ticket, double timeout_s);
int hptt_cuda_server_drain(hptt_cuda_server_t server, double timeout_s);
int hptt_cuda_server_stats(hptt_cuda_server_t server, hptt_cuda_serve_stats *stats);
int hptt_cuda_server_reset_stats(hptt_cuda_server_t server);
int hptt_cuda_server_run_poisson(hptt_cuda_server_t server, const hptt_cuda_plan_t *pool,
                                 uint32_t pool_size, double rate, double seconds,
                                 uint64_t seed, double drain_timeout_s,
                                 hptt_cuda_serve_stats *stats);
int hptt_cuda_server_destroy(hptt_cuda_server_t server);

/*
 * Tensor contraction through this library's transposes (TTGT):
 *
 *     C[labels_c] = alpha * sum_K A[labels_a] * B[labels_b] + beta * C[labels_c]
 *
 * No counterpart in the reference, which only transposes: this wraps its
 * plan usage (create_plan, exec, reset_data; README.md:48-72) around a GEMM
 * the way transpose-based contraction code calls it.  Tensors are dense and column-major like the transposes'
 * (sizes listed fastest dimension first); labels are arbitrary int32 values,
 * each at most once per tensor.  A label in A and C is an M index, in B and C
 * an N index, in A and B (not C) a summed K index, in all three a batch
 * index; C's extents come from A and B.  Not contractions (HPTT_ERR_LABELS):
 * a label of one operand alone that C lacks, a C label in neither operand,
 * a shared label with two extents.
 *
 * exec runs: A -> A-hat and B -> B-hat transposes (alpha = 1, beta = 0; each
 * skipped when the operand already has a GEMM layout), one strided-batched
 * cuBLAS GEMM into C-hat, and the output transpose C = alpha * C-hat(perm) +
 * beta * C, which reads C only when |beta| >= 1e-16 (the transposes' rule,
 * inc/hptt/impl/hptt_trans_impl.h:75-78).  When C-hat already has C's
 * layout the GEMM applies alpha and beta itself.  Label orders and layouts
 * are chosen to transpose the fewest elements.  f32 GEMMs run in full f32
 * (no reduced-precision tensor-core modes).  From the second exec on, the
 * whole sequence replays as one CUDA graph (transposes of A and B in
 * parallel branches) unless hptt_cuda_contract_set_graph(plan, 0).
 *
 *   rank_a, rank_b  1..8;  rank_c 0..8 (0: C is one element)
 *   alpha, beta     two doubles each, as for hptt_cuda_plan_create
 *   A, B, C         device pointers; never freed by the plan
 *   workspace       device memory for A-hat, B-hat, C-hat and the GEMM
 *                   library's workspace, 256-byte aligned, at least the
 *                   bytes hptt_cuda_contract_inspect reports
 *                   (HPTT_ERR_BUDGET otherwise); NULL: the plan allocates
 *                   and frees its own.
 * Like a transpose plan, one contraction plan is not executed from two host
 * threads at once; execs on different streams must not overlap (they share
 * the workspace).  destroy may be called with work in flight: it waits for
 * the device before freeing memory.
 */
typedef struct hptt_cuda_contract_s *hptt_cuda_contract_t;
typedef struct {
  uint64_t m, n, k, batch;    /* GEMM extents */
  uint64_t flops;             /* 2 m n k batch (8 m n k batch for complex) */
  uint64_t transpose_bytes;   /* bytes the transposes move per exec */
  uint64_t workspace_bytes;
  uint32_t transposes;        /* transposes per exec, 0..3 */
  uint32_t graph;             /* 1 once exec replays a captured graph */
} hptt_cuda_contract_stats;
int hptt_cuda_contract_create(int dtype, uint32_t rank_a, const uint32_t *size_a,
                              const int32_t *labels_a, uint32_t rank_b, const uint32_t *size_b,
                              const int32_t *labels_b, uint32_t rank_c,
                              const int32_t *labels_c, const double *alpha,
                              const double *beta, int complex_scalars, const void *A,
                              const void *B, void *C, void *workspace,
                              uint64_t workspace_bytes, hptt_cuda_contract_t *plan);
/* Host-only: validate, choose the layout, write its summary and the
 * workspace size (no device needed). */
int hptt_cuda_contract_inspect(int dtype, uint32_t rank_a, const uint32_t *size_a,
                               const int32_t *labels_a, uint32_t rank_b,
                               const uint32_t *size_b, const int32_t *labels_b,
                               uint32_t rank_c, const int32_t *labels_c, char *buf, size_t len,
                               uint64_t *workspace_bytes);
int hptt_cuda_contract_exec(hptt_cuda_contract_t plan);
int hptt_cuda_contract_exec_on(hptt_cuda_contract_t plan, void *stream);
int hptt_cuda_contract_reset_data(hptt_cuda_contract_t plan, const void *A, const void *B,
                                  void *C);
int hptt_cuda_contract_set_coef(hptt_cuda_contract_t plan, const double *alpha,
                                const double *beta, int complex_scalars);
int hptt_cuda_contract_set_stream(hptt_cuda_contract_t plan, void *stream);
int hptt_cuda_contract_set_graph(hptt_cuda_contract_t plan, int use_graph);
int hptt_cuda_contract_sync(hptt_cuda_contract_t plan);
int hptt_cuda_contract_info(hptt_cuda_contract_t plan, hptt_cuda_contract_stats *info);
int hptt_cuda_contract_describe(hptt_cuda_contract_t plan, char *buf, size_t len);
int hptt_cuda_contract_destroy(hptt_cuda_contract_t plan);

/* Autotune cache: the tile parameters the tuner picked, one entry per
 * (GPU name, dtype, fused rank, fused perm, size class, B read, extent
 * class floor(log2) of every fused dim).  Plans
 * created with tuning_timeout == 0 use a matching entry instead of the
 * heuristic.  The file named by the environment variable
 * HPTT_B200_TUNE_CACHE is read on first use and rewritten after every tuning
 * run.  Replaces the reference's in-plan tuning state, which lives only as
 * long as the plan (inc/hptt/plan/plan_trans.tcc:33-67); no reference
 * counterpart for persistence.
 *   load   merge the entries of a cache file (NULL: re-read the variable's)
 *   save   write every entry (NULL: to the variable's file; no-op if unset)
 *   clear  drop every entry (the variable's file is not read again)
 *   size   number of entries in *count */
int hptt_cuda_tune_cache_load(const char *path);
int hptt_cuda_tune_cache_save(const char *path);
int hptt_cuda_tune_cache_clear(void);
int hptt_cuda_tune_cache_size(uint32_t *count);

/* Static text for a status code. */
const char *hptt_cuda_status_string(int status);

/* Library version string. */
const char *hptt_cuda_version(void);

#ifdef __cplusplus
}
#endif

#endif /* HPTT_CUDA_H_ */
