/*
 * alto_b200.h -- C ABI of the B200 implementation of ALTO's hot path.
 *
 * The reference (jeewhanchoi/ALTO-stream) is a header-only C++ library used
 * in-process; it has no C ABI or FFI.  Each entry point below replaces one
 * reference interface, cited as file:line within the reference project.
 * Conventions that replace the reference's assert()/exit():
 *   - every call returns an alto_status; alto_last_error() describes the
 *     last failure on the calling thread;
 *   - all device work is ordered on the caller's CUDA stream (NULL = the
 *     legacy default stream); calls marked "synchronous" wait for it;
 *   - handles are not thread safe: use one handle from one host thread at
 *     a time;
 *   - index and size arguments are 64-bit; nonzero counts must be below 2^32;
 *     at most ALTO_MAX_MODES modes; ALTO keys are 64 or 128 bits wide.
 * There is no CPU fallback: without a usable CUDA device every call that
 * does device work returns ALTO_ERR_CUDA.
 */
#ifndef ALTO_B200_H_
#define ALTO_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALTO_MAX_MODES 8
#define ALTO_VERSION 100

typedef enum {
  ALTO_OK = 0,
  ALTO_ERR_INVALID = 1,     /* bad argument (the reference asserts)                  */
  ALTO_ERR_CUDA = 2,        /* a CUDA runtime call failed or no device is usable     */
  ALTO_ERR_NOMEM = 3,       /* device allocation failed                             */
  ALTO_ERR_NOT_SPD = 4,     /* Cholesky of a normal-equation matrix failed          */
  ALTO_ERR_UNSUPPORTED = 5, /* configuration outside the supported range            */
  ALTO_ERR_TIMEOUT = 6      /* a bounded device-side wait gave up                   */
} alto_status;

typedef enum { ALTO_F32 = 0, ALTO_BF16 = 1, ALTO_F64 = 2 } alto_dtype;

/* MTTKRP kernel variants (the reference's variants, include/alto.hpp:1349-1801,
 * re-designed for the GPU).  ALTO_MTTKRP_AUTO applies the reference's
 * selection rule (include/alto.hpp:826-848) and then the tuned choice. */
typedef enum {
  ALTO_MTTKRP_AUTO = 0,
  ALTO_MTTKRP_ATOMIC = 1,   /* vector atomics per nonzero, consecutive equal rows merged in the warp */
  ALTO_MTTKRP_STAGED = 2,   /* partition-local output rows staged in shared memory (da_mem_pull)    */
  ALTO_MTTKRP_STREAM = 3,   /* single or few output rows held in registers (mttkrp_alto_stream)     */
  ALTO_MTTKRP_SORTED = 4,   /* a row-sorted copy of the line, runs reduced in registers (op_sched)  */
  /* SORTED without atomics: runs split between lane groups are summed in a
   * fixed order afterwards, so the output repeats bit for bit from run to
   * run (float32 factors, rank 8/16/32/64/128, 16-byte aligned buffers).
   * The reference's threaded variants are not reproducible run to run. */
  ALTO_MTTKRP_DETERMINISTIC = 5
} alto_mttkrp_variant;

/* OR-ed into the variant given to alto_mttkrp_variant_run (ATOMIC or
 * SORTED): stream the line through shared memory with bulk copies
 * (cp.async.bulk, double buffered) instead of loading it directly. */
#define ALTO_MTTKRP_FEED_BULK 0x100
/* OR-ed into SORTED on a 3-mode tensor: the row-sorted walk compiled for
 * five resident blocks per SM (at most 48 registers a thread) instead of
 * four (the autotuner tries it). */
#define ALTO_MTTKRP_FEED_DENSE 0x200
/* OR-ed into SORTED on a 3-mode tensor: the five-blocks walk compiled once
 * per target mode, so the rows of the decoded records need no per-nonzero
 * mode selection (the autotuner tries it). */
#define ALTO_MTTKRP_FEED_FIXED_TARGET 0x400

/* Constraint of the CP-stream factor solves (src/constraints.cpp:39-66; the
 * reference projects LASSO onto the non-negative orthant too). */
typedef enum { ALTO_UNCONSTRAINED = 0, ALTO_NONNEG = 1, ALTO_LASSO = 2 } alto_constraint;

/* CP-ALS fit: the reference's value keeps only the diagonal of the Gram
 * Hadamard product (its Gram lower triangles are never written,
 * include/cpd.hpp:228-256); EXACT uses the full product. */
typedef enum { ALTO_FIT_REFERENCE = 0, ALTO_FIT_EXACT = 1 } alto_fit_mode;

/* A coordinate-format sparse tensor (the reference's SparseTensor,
 * include/sptensor.hpp:8-26): cidx[m] holds the nnz 0-based indices of mode
 * m, vals the nnz values.  Host or device memory. */
typedef struct {
  int nmodes;
  const uint64_t* dims;        /* host array [nmodes]                        */
  uint64_t nnz;
  const void* const* cidx;     /* host array of nmodes pointers              */
  int index_bytes;             /* 8 (uint64_t, the reference's IType) or 4   */
  const void* vals;
  alto_dtype val_dtype;        /* ALTO_F64 (the reference's FType) or F32    */
  int on_device;               /* 0: cidx/vals are host memory; 1: device    */
} alto_coo;

typedef struct alto_tensor alto_tensor;
typedef struct alto_stream_session alto_stream_session;
typedef void* alto_cuda_stream; /* a cudaStream_t */

/* ------------------------------------------------------------- library */

const char* alto_status_string(alto_status s);
const char* alto_last_error(void);
int alto_version(void);
/* Number of kernels this library launched since load (for launch audits). */
uint64_t alto_kernel_launches(void);

/* ------------------------------------------------------ the ALTO tensor */

/* The linearisation masks for a tensor shape, host only (no device work):
 * setup_packed_alto(LSB_FIRST, SHORT_FIRST), include/alto.hpp:955-1057.
 * masks: 2*nmodes words (low, high); alto_mask: 2 words; *alto_bits the
 * total.  Returns ALTO_ERR_UNSUPPORTED when the bits exceed key_bits. */
alto_status alto_compute_masks(int nmodes, const uint64_t* dims, int key_bits, uint64_t* masks,
                               uint64_t* alto_mask, int* alto_bits);

/* Linearise, sort and partition a COO tensor on the device.
 * Replaces create_alto (include/alto.hpp:436-582) when stream_mode < 0 and
 * init_salto + update_salto (include/alto.hpp:151-299) otherwise.
 * key_bits: 0 picks 64 when the index bits fit, else 128; 64 or 128 forces.
 * nprtn: the reference's partition count (prtn_ptr / prtn_intervals,
 * include/alto.hpp:1128-1226), kept for export and the staged variant. */
alto_status alto_tensor_create(const alto_coo* coo, int key_bits, int nprtn, int stream_mode,
                               alto_cuda_stream stream, alto_tensor** out);

/* Re-encode a new slice into an existing tensor, reusing its device
 * capacity (update_salto, include/alto.hpp:195-299). */
alto_status alto_tensor_update(alto_tensor* t, const alto_coo* coo, int nprtn,
                               alto_cuda_stream stream);

/* Copy the encoding to host memory, synchronous; any pointer may be NULL.
 * masks: 2*nmodes words (low, high 64 bits of each mode mask,
 * AltoTensor::mode_masks); alto_mask: 2 words; idx: 2*nnz words (the
 * reference's bit-interleaved LIT key, include/alto.hpp:513-533); vals: nnz
 * (float32 as stored, widened); perm: nnz input positions in line order;
 * prtn_ptr: nprtn+1; intervals: 2*nprtn*nmodes (start, stop), partition-major. */
alto_status alto_tensor_export(const alto_tensor* t, uint64_t* masks, uint64_t* alto_mask,
                               uint64_t* idx, double* vals, uint64_t* perm, uint64_t* prtn_ptr,
                               uint64_t* intervals);

/* Shape and encoding parameters (host outputs, any may be NULL). */
alto_status alto_tensor_info(const alto_tensor* t, int* nmodes, uint64_t* dims, uint64_t* nnz,
                             int* key_bits, int* alto_bits, int* nprtn, int* stream_mode);

/* Bytes of device memory the tensor holds. */
alto_status alto_tensor_device_bytes(const alto_tensor* t, uint64_t* bytes);

/* Keep only line entries [begin, end) of the tensor's ALTO order: one
 * GPU's shard of a sharded MTTKRP.  The shards follow the reference's
 * partition rule (prtn_alto, include/alto.hpp:1128-1160: partition p of P
 * is [min(p*ceil(nnz/P), nnz), min((p+1)*ceil(nnz/P), nnz))); each GPU runs
 * its MTTKRP into a full-size output and an all-reduce (sum) gives the
 * tensor's MTTKRP.  Dims, masks and the key layout are unchanged; tiles,
 * intervals and partitions are rebuilt for the kept entries. */
alto_status alto_tensor_restrict(alto_tensor* t, uint64_t begin, uint64_t end, alto_cuda_stream stream);

alto_status alto_tensor_destroy(alto_tensor* t); /* destroy_alto, include/alto.hpp:584-604 */

/* --------------------------------------------------------------- MTTKRP */

/* out (rows dims[mode] x rank, row-major float32, device) receives the
 * mode-`mode` MTTKRP of the tensor with the factor matrices factors[m]
 * (device, dims[m] x rank row-major, dtype fdtype = ALTO_F32 or ALTO_BF16;
 * factors[mode] is not read).  accumulate != 0 adds to out as the reference
 * does (it accumulates into factors[target_mode]); 0 overwrites.
 * Replaces mttkrp_alto_par (include/alto.hpp:902-908). */
alto_status alto_mttkrp(alto_tensor* t, int mode, const void* const* factors, alto_dtype fdtype,
                        int rank, float* out, int accumulate, alto_cuda_stream stream);

/* As alto_mttkrp with an explicit kernel variant (for tests and tuning). */
alto_status alto_mttkrp_variant_run(alto_tensor* t, int mode, const void* const* factors,
                                    alto_dtype fdtype, int rank, float* out, int accumulate,
                                    alto_mttkrp_variant variant, alto_cuda_stream stream);

/* Project autotuner: time every applicable variant once per mode with these
 * factors (rank, fdtype) and make ALTO_MTTKRP_AUTO use the fastest.
 * variants (may be NULL) receives the choice per mode.  Synchronous; call
 * it outside stream capture.  The reference fixes its choice at compile
 * time (rank/mode specialisation, include/alto.hpp:826-900). */
alto_status alto_mttkrp_autotune(alto_tensor* t, const void* const* factors, alto_dtype fdtype,
                                 int rank, alto_cuda_stream stream, alto_mttkrp_variant* variants);

/* The variant ALTO_MTTKRP_AUTO resolves to for this tensor, mode and rank. */
alto_status alto_mttkrp_choose(const alto_tensor* t, int mode, int rank, alto_dtype fdtype,
                               alto_mttkrp_variant* variant);

/* Host-buffer MTTKRP, the drop-in for mttkrp_alto_par's calling convention:
 * factors_host[m] are dims[m] x rank float64 host arrays and
 * factors_host[mode] is accumulated into, as in the reference.  Copies in,
 * computes in float32 on the device, copies out; synchronous. */
alto_status alto_mttkrp_host(alto_tensor* t, int mode, double* const* factors_host, int rank,
                             alto_cuda_stream stream);

/* alto_mttkrp_host for callers that change few factors between calls (a
 * CP-ALS loop rewrites one factor per mode step): bit m of `changed` says
 * factors_host[m] was modified on the host since this thread's previous
 * host-buffer MTTKRP.  A factor with its bit clear, at the same host
 * address and size as in that call, is not copied again (the device keeps
 * the copy it last sent or returned); factors_host[mode] is still
 * accumulated into and copied back.  The first call copies everything.
 * Same results as alto_mttkrp_host. */
alto_status alto_mttkrp_host_changed(alto_tensor* t, int mode, double* const* factors_host, int rank,
                                     uint32_t changed, alto_cuda_stream stream);

/* ------------------------------------------------------ dense helpers */

/* G = U^T U in float64 (rank x rank, full symmetric, row-major, device) of a
 * float32 factor U (rows x rank, row-major, device): update_gram / mat_aTa
 * (src/gram.cpp:29-41, src/matrix.cpp:252-267; the reference's dsyrk fills
 * only the upper triangle, here both are written).  rank <= 128.  The
 * per-block partial sums live in device memory the library allocates and
 * keeps for later calls. */
alto_status alto_gram(const float* U, uint64_t rows, int rank, double* G, alto_cuda_stream stream);

/* alto_gram for callers that cannot allocate device memory (a process whose
 * pool owns all of HBM, an allocator that is off limits inside graph
 * capture or a real-time loop, an embedder that may not call cudaMalloc /
 * cudaFree).  It has no counterpart in the reference.  Same arguments and
 * result as alto_gram, but rank <= 64 (ALTO_ERR_UNSUPPORTED beyond) and no
 * allocation: the partial sums live in a fixed 2 MiB device array inside
 * this library, present on every GPU that loads it until the process
 * exits.  The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) and keeps it for the life of the process, so make
 * that call before any stream capture, and do not call this entry point on
 * a device after cudaDeviceReset of it (the kept address would be stale;
 * the rest of the library has the same rule for its cached buffers).  All calls
 * share the array: calls that may overlap on the GPU (different streams or
 * host threads without ordering) race and must be serialised by the caller. */
alto_status alto_gram_noalloc(const float* U, uint64_t rows, int rank, double* G,
                              alto_cuda_stream stream);

/* --------------------------------------------------------------- CP-ALS */

/* CP-ALS on the device (cpd_alto, include/cpd.hpp:47-191).  U_host[n]
 * (dims[n] x rank float64) and lambda_host (rank) hold the initial model on
 * entry and the result on exit.  Factors are stored on the device as
 * storage (ALTO_F32 or ALTO_BF16); MTTKRP accumulates in float32; Grams,
 * Cholesky, solves and fit are float64.  fits (max_iters, may be NULL)
 * receives the per-iteration residual; *iters the iterations run.
 * Synchronous. */
alto_status alto_cpd_als(alto_tensor* t, int rank, double* const* U_host, double* lambda_host,
                         int max_iters, double epsilon, alto_fit_mode fit_mode,
                         alto_dtype storage, double* fits, int* iters, alto_cuda_stream stream);

/* ------------------------------------------------------------ CP-stream */

/* A CP-stream session keeps the model, previous model, Grams and ADMM state
 * resident on the device between time batches (cpstream,
 * src/streaming_cpd.cpp:26-366 with cpstream_alto_iter :1198-1519).
 * forgetting: the temporal Gram decay (the reference hard-codes 0.99,
 * src/streaming_cpd.cpp:18). */
alto_status alto_stream_open(int nmodes, int stream_mode, int rank, alto_constraint constraint,
                             double forgetting, int max_inner_iters, double epsilon,
                             alto_cuda_stream stream, alto_stream_session** out);

/* Process one time batch.  Rows the model gains take their initial values
 * from init_vals (host, n_init values consumed in order: mode 0's new rows,
 * then mode 1's, ...; the reference draws them from rand(),
 * src/kruskal_model.cpp:101-178); missing values are zero.  *inner_iters
 * (may be NULL) receives the inner iterations run.  Synchronous. */
alto_status alto_stream_push(alto_stream_session* s, const alto_coo* batch,
                             const double* init_vals, uint64_t n_init, int* inner_iters);

/* Copy mode m of the current model (dims[m] x rank float64) to host memory;
 * for the stream mode this is the concatenated time factor (every batch's
 * time rows).  rows receives the row count.  Synchronous. */
alto_status alto_stream_factor(alto_stream_session* s, int mode, double* host_out,
                               uint64_t* rows);
alto_status alto_stream_lambda(alto_stream_session* s, double* host_out);

/* The streaming model of a session (the reference's -l cpstream_alto |
 * spcpstream_alto, src/main.cpp:158-165; cpstream(..., use_spcpstream, ...),
 * src/streaming_cpd.cpp:26).  CP-stream solves every row of every mode in
 * each inner iteration and applies the constraint; spCP-stream
 * (spcpstream_alto_iter, src/streaming_cpd.cpp:466-1085) solves only the
 * rows a batch touches and moves the others in closed form, and, as in the
 * reference, does not use the constraint.  Set before the first push. */
typedef enum { ALTO_MODEL_CPSTREAM = 0, ALTO_MODEL_SPCPSTREAM = 1 } alto_stream_model;
alto_status alto_stream_set_model(alto_stream_session* s, alto_stream_model model);

/* How alto_stream_push issues a batch's inner iterations (the reference's
 * loop, src/streaming_cpd.cpp:1240-1482).  enable = 1 (the default): all
 * of them as one launch of a CUDA graph captured once per session and
 * relaunched for every batch, whose while nodes run the inner loop and the
 * ADMM sweeps with the stopping tests on the device (sizes and pointers
 * read from device memory).  enable = 0: every launch directly, one host
 * synchronisation per inner iteration.  Both give identical results. */
alto_status alto_stream_set_graph(alto_stream_session* s, int enable);

/* Where a session's pushes spent their time, summed over its pushes:
 * out[0] pushes; out[1] host ms preparing batches (model growth, the
 * batch's encoding and row-sorted copies, Grams); out[2] host ms from the
 * inner iterations' launch until their outcome is on the host; out[3]
 * device ms of the inner iterations (CUDA events around their launch);
 * out[4] host ms finishing (forgetting, copies, the time row out); out[5]
 * inner iterations; parts of out[1]: out[6] host ms growing the model
 * (reallocations, new rows), out[7] encoding the batch, out[8] building its
 * row-sorted copies. */
alto_status alto_stream_stats(const alto_stream_session* s, double out[9]);
/* cpd_error(X, M), src/streaming_cpd.cpp:368-464: the relative residual
 * ||X - M|| / ||X|| of the session's current model (unit weights, as
 * cpd_error sets them) against a COO tensor X in the session's indexing
 * (host or device).  X's time indices address the last X->dims[t] rows of
 * the model's time factor: the whole factor for the whole tensor (the
 * reference's final "fit error" is err^2), the last `previous` rows for
 * alto_slicer_stream_prev(previous) as compute_errorsq does
 * (src/streaming_cpd.cpp:1521-1532).  Model rows past the session's dims
 * are zero.  Synchronous. */
alto_status alto_stream_error(alto_stream_session* s, const alto_coo* X, double* err);
alto_status alto_stream_close(alto_stream_session* s);

/* ---------------------------------------------------------- tensor files */

/* The reference's FileFormat (include/sptensor.hpp:29-32). */
typedef enum { ALTO_FILE_TEXT = 0, ALTO_FILE_BINARY = 1 } alto_file_format;

/* A COO tensor read from a file into device memory (uint64 indices,
 * float64 values: the reference's IType and FType). */
typedef struct alto_dcoo alto_dcoo;

/* ImportSparseTensor(path, format, &X, zero_based), src/sptensor.cpp:160-249.
 * Text (.tns): whitespace-separated indices then a value per line, '#'
 * comments, 1-based unless zero_based; the mode count is the first line's
 * token count minus one and dims[m] the largest index (+1 when zero_based),
 * exactly as the reference reads them (src/sptensor.cpp:74-158).  The file
 * is streamed into HBM and parsed there; values equal the C library's
 * strtod bit for bit.  Binary: uint64 nmodes, dims[nmodes], nnz, the index
 * arrays mode by mode, float64 values.  An unreadable file, a file without
 * nonzeros or a short binary file is ALTO_ERR_INVALID.  The read's working
 * buffers (about the file's size plus 8 bytes per line) come from a device
 * memory pool the library keeps for later reads and slicers until the
 * process exits.  Synchronous. */
alto_status alto_read_tensor(const char* path, alto_file_format format, int zero_based,
                             alto_cuda_stream stream, alto_dcoo** out);
/* A device view of the tensor (on_device 1, index_bytes 8, ALTO_F64), valid
 * until alto_dcoo_destroy; it can be given to alto_tensor_create,
 * alto_slicer_create and alto_stream_push. */
alto_status alto_dcoo_view(const alto_dcoo* d, alto_coo* view);
/* Timings of the read: host file reading and copies (read_ms), device
 * parse (parse_ms, text only); the file's size; how many values the device
 * left to the C library's strtod.  Any pointer may be NULL. */
alto_status alto_dcoo_stats(const alto_dcoo* d, double* read_ms, double* parse_ms, uint64_t* file_bytes,
                            uint64_t* host_values);
/* The tensor in host memory, as ImportSparseTensor leaves it: cidx
 * [nmodes][nnz] uint64, vals [nnz] float64 (either may be NULL).  Synchronous. */
alto_status alto_dcoo_to_host(const alto_dcoo* d, uint64_t* cidx, double* vals);
alto_status alto_dcoo_destroy(alto_dcoo* d);

/* ExportSparseTensor(path, format, X), src/sptensor.cpp:22-72, from a host
 * or device COO: text lines of "%llu " (index + 1) per mode and "%g\n" of
 * the value, formatted on all host cores; or the binary layout above.
 * Synchronous. */
alto_status alto_write_tensor(const char* path, alto_file_format format, const alto_coo* coo);

/* ---------------------------------------------------------- stream slicer */

/* The reference's StreamingSparseTensor (include/streaming_sptensor.hpp:10-44)
 * on the device.  A whole tensor is sorted by the stream mode, then the
 * following modes cyclically (tt_sort, src/sort.cpp:477-519), and every
 * other mode is relabelled in first-seen order; batches of whole time steps
 * are then cut from it.  Batches are device views (index_bytes 4, the input's
 * value type, on_device 1) that alto_stream_push takes directly. */
typedef struct alto_slicer alto_slicer;

/* StreamingSparseTensor(sp, stream_mode), src/streaming_sptensor.cpp:69-125.
 * coo: host or device COO; dims[m] < 2^32, nmodes * (nnz + 1) < 2^32 and
 * the bits of all dims <= 128 (ALTO_ERR_UNSUPPORTED otherwise); an index
 * outside its mode is ALTO_ERR_INVALID.  Construction's working buffers
 * (about 60 bytes per nonzero) come from the library's device memory pool
 * (kept for later calls, as alto_read_tensor's).  Synchronous. */
alto_status alto_slicer_create(const alto_coo* coo, int stream_mode, alto_cuda_stream stream,
                               alto_slicer** out);
/* next_dynamic_batch(nnz_threshold, timeslice_limit), :196-264: grow the
 * batch by whole time steps while it holds fewer than nnz_threshold
 * nonzeros and fewer than timeslice_limit steps.  *batch receives views of
 * s's device arrays (consecutive batches are consecutive ranges of them),
 * valid until alto_slicer_destroy; its host dims and cidx arrays belong to
 * s and are overwritten by the next call.  The stream-mode indices are
 * local to the batch.
 * *got = 0 once every nonzero was returned (the reference returns NULL).
 * A run of time steps without nonzeros gives a batch with nnz 0, as the
 * reference does when built without assertions (it asserts nnz > 0). */
alto_status alto_slicer_next(alto_slicer* s, uint64_t nnz_threshold, uint64_t timeslice_limit,
                             alto_coo* batch, int* got);
/* Every remaining batch at once: the cuts repeated alto_slicer_next calls
 * would make, with the batch-local time indices of all of them written by
 * one kernel (no counterpart in the reference, whose slicer only iterates).
 * *nbatches receives the count; alto_slicer_batch then gives each view. */
alto_status alto_slicer_cut_all(alto_slicer* s, uint64_t nnz_threshold, uint64_t timeslice_limit,
                                uint64_t* nbatches);
/* Batch b of the last alto_slicer_cut_all, as alto_slicer_next returns it
 * (its cidx array is overwritten by the next call on s). */
alto_status alto_slicer_batch(alto_slicer* s, uint64_t b, alto_coo* out);
/* last_batch(), :266-269. */
alto_status alto_slicer_last_batch(const alto_slicer* s, int* last);
/* stream_prev(previous), :284-327: the nonzeros of the last `previous` time
 * steps returned so far, time indices relative to the first of them; other
 * dims as of the last batch.  Valid until the next stream_prev call. */
alto_status alto_slicer_stream_prev(alto_slicer* s, uint64_t previous, alto_coo* out, int* got);
/* The whole tensor as the reference's StreamingSparseTensor holds it after
 * construction: sorted, relabelled, global time indices, the input dims
 * (device view, valid until alto_slicer_destroy; for alto_stream_error). */
alto_status alto_slicer_tensor(const alto_slicer* s, alto_coo* out);
/* The original index of every label of `mode` (the Permutation iperms the
 * reference keeps, :92-124) to host memory; *count receives how many
 * (host_out may be NULL to ask for the count). */
alto_status alto_slicer_iperm(alto_slicer* s, int mode, uint64_t* host_out, uint64_t* count);
alto_status alto_slicer_destroy(alto_slicer* s);

/* -------------------------------------------------------------- serving */

/* A server for many independent CP-stream tensors (the reference has none;
 * it runs one stream's slices one at a time, src/streaming_cpd.cpp:26-366).
 * Slices are submitted as host COO batches and processed by `workers`
 * threads, each on its own CUDA stream, so the updates of different streams
 * overlap on the GPU; a stream's own slices run in submission order.  Each
 * stream's model, Grams and ADMM state stay on the device.  Streams are
 * admitted while the sum of their reserved footprints stays within
 * hbm_budget_bytes; a stream that does not fit waits, with its slices
 * queued, until earlier streams close. */
typedef struct alto_server alto_server;

typedef struct {
  int nmodes;
  int stream_mode;
  int rank;
  alto_constraint constraint;
  double forgetting;
  int max_inner_iters;
  double epsilon;
  alto_stream_model model;  /* ALTO_MODEL_CPSTREAM or ALTO_MODEL_SPCPSTREAM */
} alto_stream_config;

typedef struct {
  uint64_t submitted, completed;
  double p50_ms, p99_ms, max_ms;  /* slice latency, submission to completion, over
                                     the last 2^20 completed slices */
  double slices_per_s;            /* completed slices over first submission .. last completion */
  uint64_t reserved_bytes;
  int admitted_streams, pending_streams;
  /* where the time went (host clock, summed over threads): slice
   * preparation on the workers, group steps on the scheduler (launch to
   * states read back), finishing on the workers; group steps run and the
   * slices they covered (their ratio: the mean slices per step) */
  double prepare_ms, step_ms, finish_ms;
  uint64_t steps, step_slices;
} alto_serving_stats;

alto_status alto_server_create(uint64_t hbm_budget_bytes, int workers, alto_server** out);
/* Open a stream; max_dims (nmodes) and max_slice_nnz bound its footprint
 * estimate for admission.  *sid receives its id; it may wait for admission. */
alto_status alto_server_open(alto_server* s, const alto_stream_config* cfg, const uint64_t* max_dims,
                             uint64_t max_slice_nnz, int* sid);
/* Queue one time batch (copied; host memory).  init_vals as alto_stream_push. */
alto_status alto_server_submit(alto_server* s, int sid, const alto_coo* batch, const double* init_vals,
                               uint64_t n_init, uint64_t* ticket);
/* Wait for one slice; its status, inner iterations and latency.  A ticket is
 * handed back once: after wait (or a poll that reports it done) returns it,
 * the server forgets it and a second wait or poll is ALTO_ERR_INVALID.  A
 * slice dropped by alto_server_close before its stream was admitted ends
 * with ALTO_ERR_INVALID. */
alto_status alto_server_wait(alto_server* s, uint64_t ticket, int* inner_iters, double* latency_ms);
/* The same without waiting: *done = 0 while the slice is queued or running
 * (ALTO_OK), else 1 with alto_server_wait's outputs and status (and the
 * ticket is handed back, as by wait). */
alto_status alto_server_poll(alto_server* s, uint64_t ticket, int* done, int* inner_iters, double* latency_ms);
/* Wait until every admitted stream has processed all its slices. */
alto_status alto_server_drain(alto_server* s);
alto_status alto_server_stats(alto_server* s, alto_serving_stats* out);
/* A stream's factor (as alto_stream_factor) once its queued slices are done. */
alto_status alto_server_factor(alto_server* s, int sid, int mode, double* host_out, uint64_t* rows);
/* Finish a stream's queued slices, free its device state, admit waiting
 * streams.  A stream not yet admitted has its queued slices dropped: their
 * tickets finish with ALTO_ERR_INVALID, waking any waiter. */
alto_status alto_server_close(alto_server* s, int sid);
alto_status alto_server_destroy(alto_server* s);

#ifdef __cplusplus
}
#endif
#endif /* ALTO_B200_H_ */
