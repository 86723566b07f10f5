/*
 * fgkl_b200: the PairHMM / PD-HMM read-versus-haplotype likelihood path of fulcrumgenomics/fgkl,
 * rebuilt for NVIDIA B200 (sm_100a), behind a plain C ABI.
 *
 * Every entry point takes plain pointers and sizes, returns 0 (FGKL_OK) or a negative FGKL_E_*
 * code, and never aborts; fgkl_last_error() gives the calling thread's last message. Likelihoods
 * are log10 values written row-major, out[read * num_haplotypes + haplotype], in the caller's
 * read and haplotype order, exactly as fgkl's PairHmm::compute_log10_likelihoods
 * (crates/pairhmm/src/lib.rs:270-293) and its JNI entry points (crates/jni/src/lib.rs:159-254).
 *
 * Threading: any number of threads may call concurrently. The per-call entry points use a
 * context private to the calling thread (created on first use), mirroring fgkl's thread-local
 * workspaces (crates/pairhmm/src/kernel.rs:144-163). Calls from several threads that meet are run
 * as one batch on an engine kept for combining (fgkl_set_call_combining). Explicit contexts must not
 * be shared between threads without external locking.
 */
#ifndef FGKL_B200_H
#define FGKL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes; the first five mirror fgkl's Error enum (crates/pairhmm/src/lib.rs:303-323) ---- */
#define FGKL_OK 0
#define FGKL_E_EMPTY_READ (-1)                  /* Error::EmptyRead */
#define FGKL_E_MISMATCHED_READ_ARRAYS (-2)      /* Error::MismatchedReadArrays */
#define FGKL_E_EMPTY_HAPLOTYPE (-3)             /* Error::EmptyHaplotype */
#define FGKL_E_MISMATCHED_HAPLOTYPE_ARRAYS (-4) /* Error::MismatchedHaplotypeArrays */
#define FGKL_E_OUTPUT_LENGTH (-5)               /* Error::OutputLength */
#define FGKL_E_BAD_OFFSETS (-6)                 /* offset table checks of crates/jni/src/lib.rs:343-363 */
#define FGKL_E_INVALID_ARGUMENT (-7)            /* NULL pointer or negative size */
#define FGKL_E_UNSUPPORTED (-8)                 /* an input outside what an entry point takes (adjoint: a haplotype over 2^24 bases; allocation-free entry: its limits) */
#define FGKL_E_NO_DEVICE (-9)                   /* no CUDA device, or not an sm_100 part */
#define FGKL_E_CUDA (-10)                       /* CUDA runtime error (message in fgkl_last_error) */
#define FGKL_E_OUT_OF_MEMORY (-11)              /* a device or page-locked host allocation failed; the caller may retry smaller */
#define FGKL_E_EMPTY_SEQUENCE (-12)             /* Smith-Waterman: fgkl_smithwaterman::Error::EmptySequence */

/* How to compute (crates/pairhmm/src/lib.rs:211-238). */
typedef struct fgkl_config {
  int32_t double_precision; /* 0: FP32 with FP64 recomputation of lost pairs (Precision::Float) */
  int32_t double_fallback;  /* recompute lost pairs; 0 leaves them NaN (lib.rs:218-222) */
  int32_t share_suffixes;   /* suffix sharing for the plain PairHMM (lib.rs:223-226) */
} fgkl_config;

/* Counters of one call. */
typedef struct fgkl_stats {
  uint64_t fallback_pairs;    /* pairs lost by the first pass (PairHmm::fallback_pairs, lib.rs:263-268) */
  uint64_t rescue_reads;      /* (read, distinct haplotype) pairs recomputed in FP64 without sharing */
  uint64_t nominal_cells;     /* Σ over regions of Σ read lengths x Σ haplotype lengths */
  uint64_t computed_cells;    /* forward + backward DP cells the first pass computed */
  uint64_t forward_cells;
  uint64_t backward_cells;
  uint64_t prefix_only_cells; /* forward cells with prefix sharing alone */
  uint64_t kernel_launches;   /* kernels launched by the call's run phase */
  double host_plan_ms;        /* host time: sorting, planning, program emission */
  double host_pack_ms;        /* host time: packing the batch into pinned staging */
  double host_upload_ms;      /* host time: enqueueing the uploads */
  double host_fetch_ms;       /* host time: waiting for the kernels and copying results out */
} fgkl_stats;

/* The five read arrays of one call, concatenated, delimited by `offsets` (num_reads + 1 entries,
 * starting at 0, non-decreasing, ending at the array length), as the JNI boundary passes them. */
typedef struct fgkl_reads {
  const uint8_t* bases;   int64_t bases_len;
  const uint8_t* quals;   int64_t quals_len;
  const uint8_t* ins_gop; int64_t ins_gop_len;
  const uint8_t* del_gop; int64_t del_gop_len;
  const uint8_t* gcp;     int64_t gcp_len;
  const int32_t* offsets; int64_t offsets_len;
} fgkl_reads;

/* Concatenated haplotypes; `flags` (same length as `bases`) only for the PD-HMM. */
typedef struct fgkl_haplotypes {
  const uint8_t* bases;   int64_t bases_len;
  const uint8_t* flags;   int64_t flags_len;
  const int32_t* offsets; int64_t offsets_len;
} fgkl_haplotypes;

/*
 * Per-call PairHMM: the drop-in for
 *   Java_com_fulcrumgenomics_fgkl_pairhmm_FgklPairHmm_computeNative  (crates/jni/src/lib.rs:159-195)
 * which builds PairHmm::new(&config(double)) (lib.rs:247-251) and calls
 * compute_log10_likelihoods (lib.rs:270-293). `out_len` must be num_reads * num_haplotypes.
 */
int fgkl_pairhmm_compute(const fgkl_reads* reads, const fgkl_haplotypes* haps, int32_t double_precision,
                         double* out, int64_t out_len);

/* As fgkl_pairhmm_compute with an explicit Config (lib.rs:211-238) and call counters. */
int fgkl_pairhmm_compute_config(const fgkl_reads* reads, const fgkl_haplotypes* haps, const fgkl_config* config,
                                double* out, int64_t out_len, fgkl_stats* stats);

/*
 * Per-call PD-HMM: the drop-in for
 *   Java_com_fulcrumgenomics_fgkl_pdhmm_FgklPdHmm_computeNative  (crates/jni/src/lib.rs:206-254)
 * (PdPairHmm::compute_log10_likelihoods, crates/pairhmm/src/pd.rs:251-279).
 */
int fgkl_pdhmm_compute(const fgkl_reads* reads, const fgkl_haplotypes* haps, int32_t double_precision,
                       double* out, int64_t out_len);
int fgkl_pdhmm_compute_config(const fgkl_reads* reads, const fgkl_haplotypes* haps, const fgkl_config* config,
                              double* out, int64_t out_len, fgkl_stats* stats);

/*
 * Combining of concurrent per-call requests (no counterpart in the reference, whose calls each run
 * on the calling thread, crates/jni/src/lib.rs:5-9). The four per-call functions above accept any
 * number of concurrent callers, as fgkl's do.
 *
 * A call made while other threads' calls wait joins them. The first caller to find fewer than
 * `max_batches` batches in flight takes every waiting request of its kind (same entry point and
 * the same three config flags). It runs them as one batch and writes each caller's results; the
 * others wait for theirs.
 *
 * Guarantees:
 * - Results are bit-identical to separate calls.
 * - A failed batch is retried as separate calls, each on its own thread, so every caller gets its
 *   own status and fgkl_last_error.
 * - Calls that ask for stats always run alone.
 *
 * Each of the max_batches batches in flight runs on an engine of its own, kept for the process.
 * max_batches = 0 runs every call alone. The default is 2 and the largest value is 8. Returns the
 * previous value, or FGKL_E_INVALID_ARGUMENT for a value outside 0..8.
 */
int fgkl_set_call_combining(int32_t max_batches);

/* Combined batches of two or more requests run since the library loaded, and the requests they
 * held. */
int fgkl_call_combining_stats(uint64_t* batches, uint64_t* requests);

/* Failure injection (no counterpart in the reference; its Rust allocator aborts instead). From now on
 * every call that needs a device or page-locked host buffer larger than `bytes` fails with
 * FGKL_E_OUT_OF_MEMORY, as if the device could not hold it, whether or not the library already holds
 * a buffer that large; so a caller's handling of the error can be exercised without exhausting a
 * real device. Buffers already held are kept, and a call that fails leaves its engine or context
 * usable for later calls. `bytes` = 0 removes the limit. Process-wide; returns the previous limit, or
 * FGKL_E_INVALID_ARGUMENT when negative. */
int64_t fgkl_set_allocation_limit(int64_t bytes);

/* Name of the backend, the analogue of backendNative (crates/jni/src/lib.rs:149-156). */
const char* fgkl_backend(void);

/* The calling thread's last error message ("" when none). */
const char* fgkl_last_error(void);

/* ---- batched form: many regions, one planned upload, persistent launches ---- */

typedef struct fgkl_context fgkl_context;

/* Regions concatenated: region g owns region_reads[g] consecutive reads and region_haps[g]
 * consecutive haplotypes; its output block of region_reads[g] x region_haps[g] likelihoods
 * follows the previous region's. Offsets are byte offsets (total + 1 entries, starting at 0). */
typedef struct fgkl_batch {
  int32_t num_regions;
  const int32_t* region_reads;
  const int32_t* region_haps;
  const uint8_t* bases;
  const uint8_t* quals;
  const uint8_t* ins_gop;
  const uint8_t* del_gop;
  const uint8_t* gcp;
  const int64_t* read_offsets;
  const uint8_t* hap_bases;
  const uint8_t* hap_flags; /* NULL for the plain PairHMM; else per-base PD flags */
  const int64_t* hap_offsets;
} fgkl_batch;

/* A context on `device`; `stream` is a cudaStream_t to run its kernels on, or NULL for a private
 * stream. Each context copies on a private copy stream of its own. To stream batches back to back,
 * give two contexts the same stream and alternate: prepare and run batch k+1 on one, then fetch
 * batch k from the other. The host planning of k+1 and its upload overlap the kernels of k, and the
 * batches' kernels run one after another on the shared stream. */
fgkl_context* fgkl_context_create(int32_t device, void* stream);
void fgkl_context_destroy(fgkl_context* ctx);

/* Validates and plans the batch on the host and uploads it on the context's copy stream. Waits for
 * this context's previous batch only (its kernels and copies), never for other work on the stream.
 * The batch's host arrays may be reused once it returns. Read arrays in page-locked memory
 * (cudaMallocHost, cudaHostAlloc, cudaHostRegister) are uploaded from where they lie, and the call
 * waits for that upload. Others are first copied to the context's pinned staging. */
int fgkl_batch_prepare(fgkl_context* ctx, const fgkl_batch* batch, const fgkl_config* config);
/* Enqueues the kernels of the prepared batch on the context's stream, after its upload, without
 * waiting. The launch sequence is captured into a CUDA graph, updated in place for later batches. */
int fgkl_batch_run(fgkl_context* ctx);
/* Copies the likelihoods (Σ reads x haplotypes) and counters back once the batch's kernels are done,
 * and waits for that copy (not for later work on the stream). A page-locked `out` receives the
 * results directly; any other goes through the context's pinned staging. */
int fgkl_batch_fetch(fgkl_context* ctx, double* out, int64_t out_len, fgkl_stats* stats);
/* prepare + run + fetch. */
int fgkl_batch_compute(fgkl_context* ctx, const fgkl_batch* batch, const fgkl_config* config, double* out,
                       int64_t out_len, fgkl_stats* stats);
/* Number of likelihoods the prepared batch produces. */
int64_t fgkl_batch_output_len(const fgkl_context* ctx);

/* Launch configuration of a context's batched form (the autotuner's search space). */
typedef struct fgkl_tuning {
  int32_t streams;          /* streams the launches of one pass spread over, 1-8 (1: one after another) */
  int32_t grid_percent;     /* each first-pass persistent grid, % of the kernel's resident-block limit, 10-100 */
  int32_t reads_per_warp;   /* FP32 PD-HMM reads of at most 248 bases: 2 (FP32x2 pairs, the default) or 1 */
  int32_t rows_extra;       /* tile shape: 1 runs plain FP32 reads one rows-per-lane step above the fewest
                               that hold them (0, the default: the fewest) */
  int32_t warps_per_block;  /* tile shape: warps per block of the FP32 first-pass kernels, 1, 2 or 4 (default) */
  double ms;                /* autotuner: median device time of one run of the batch with this configuration */
} fgkl_tuning;

/* Autotuner. Plans `batch` once per candidate configuration and times its kernels with CUDA events:
 * one untimed run, then the median of `repeats` runs. The candidates: streams in {1, 2, 4, 8} x grid
 * in {100, 90, 75, 60} % (two reads per warp, default tile shape); for an FP32 PD-HMM batch also one
 * read per warp at 4 and 8 streams, full grids; then, from the fastest so far, the tile shapes 1 and 2
 * warps per block and, for a plain FP32 batch, one rows-per-lane step up. No configuration changes a
 * result bit. It keeps the fastest for the context's later batches and leaves `batch` prepared with
 * it. `tried` (may be NULL) receives up to `tried_cap` candidates in the order they ran, and
 * `n_tried` their count. Host-synchronous; a batch that represents the caller's workload (a sample of
 * it will do) gives the configuration that workload runs fastest with. */
int fgkl_context_autotune(fgkl_context* ctx, const fgkl_batch* batch, const fgkl_config* config, int32_t repeats,
                          fgkl_tuning* chosen, fgkl_tuning* tried, int32_t tried_cap, int32_t* n_tried);
/* Sets or reads a context's launch configuration directly (applies from the next prepare). */
int fgkl_context_set_tuning(fgkl_context* ctx, const fgkl_tuning* tuning);
int fgkl_context_get_tuning(const fgkl_context* ctx, fgkl_tuning* tuning);

/* Per-launch timing for measurement. With profiling on, fgkl_batch_run issues its launches directly
 * (no CUDA graph), one after another on the context's stream instead of concurrently, with CUDA
 * events around each, so each is timed alone; fgkl_batch_launch_profile
 * waits and reports every first-pass and recomputation launch of the last run: kernel kind
 * (0 packed FP32, 1 FP32, 2 FP64, 3 PD FP32, 4 PD FP64), rows per lane, tasks, blocks, whether it is
 * a recomputation launch, the forward and backward DP cells its tasks compute, and its duration. */
typedef struct fgkl_launch_profile {
  int32_t kind;
  int32_t rows;
  int32_t tasks;
  int32_t blocks;
  int32_t recomputation;
  uint64_t forward_cells;
  uint64_t backward_cells;
  float ms;
} fgkl_launch_profile;
int fgkl_context_profile(fgkl_context* ctx, int32_t on);
int fgkl_batch_launch_profile(fgkl_context* ctx, fgkl_launch_profile* out, int32_t max, int32_t* count);

/* ---- adjoint: gradients for fitting the indel and base-error model (no counterpart in the reference) ----
 *
 * d(Σ over every read x haplotype pair of log10 L)/d(parameter) for each read position's
 * continuous parameters: insertion and deletion gap-open probabilities dI, dD (fgkl's MI, MD),
 * gap continuation eps (II = DD = eps, IM = 1 - eps) and base error e (priors 1 - e and e / 3),
 * with MM = 1 - dI - dD. fgkl's quantized match-to-match table (crates/pairhmm/src/model.rs:43-45)
 * agrees with 1 - dI - dD to about 1e-6 but is not differentiable, hence this parameterisation.
 * Haplotype bytes compare as bytes, N matching everything (reference.rs:20-64).
 *
 * Computed with FP32 forward and backward values and FP32 products, summed per read position over
 * 32 columns at a time and accumulated in FP64; a read whose FP32 likelihood falls below 1e-28
 * against any haplotype is recomputed in FP64 (`fp64_reads` counts them). double_precision = 1 runs
 * everything in FP64. The likelihoods (log10 L per pair, row-major per region as fgkl_batch_fetch)
 * come out too. Row checkpointing: the backward values are never stored per cell; the backward
 * sweep saves its state every few columns and each block of columns is recomputed just before the
 * forward sweep uses it, so memory grows with the pair's columns / 8, not its cells. Reads of any
 * length (longer than 620 bases: strip-mined over blocks of 256 rows). The context's stream is
 * used. */
typedef struct fgkl_adjoint_batch {
  int32_t num_regions;
  const int32_t* region_reads;
  const int32_t* region_haps;
  const uint8_t* bases;
  const int64_t* read_offsets;      /* total reads + 1 */
  const double* gap_open_ins;       /* dI per read position */
  const double* gap_open_del;       /* dD */
  const double* gap_continuation;   /* eps */
  const double* base_error;         /* e */
  const uint8_t* hap_bases;
  const int64_t* hap_offsets;       /* total haplotypes + 1 */
} fgkl_adjoint_batch;

int fgkl_adjoint_prepare(fgkl_context* ctx, const fgkl_adjoint_batch* batch, int32_t double_precision);
/* Enqueues the adjoint kernels on the context's stream; `launches` (may be NULL) receives their count. */
int fgkl_adjoint_run(fgkl_context* ctx, uint64_t* launches);
/* Waits and copies out the likelihoods and the four per-position gradient arrays. */
int fgkl_adjoint_fetch(fgkl_context* ctx, double* log10_out, int64_t out_len, double* grad_gap_open_ins,
                       double* grad_gap_open_del, double* grad_gap_continuation, double* grad_base_error, int64_t grad_len,
                       uint64_t* fp64_reads);
/* prepare + run + fetch. */
int fgkl_adjoint_compute(fgkl_context* ctx, const fgkl_adjoint_batch* batch, int32_t double_precision, double* log10_out,
                         int64_t out_len, double* grad_gap_open_ins, double* grad_gap_open_del, double* grad_gap_continuation,
                         double* grad_base_error, int64_t grad_len, uint64_t* fp64_reads);
int64_t fgkl_adjoint_output_len(const fgkl_context* ctx);
int64_t fgkl_adjoint_grad_len(const fgkl_context* ctx);

/* ---- Smith-Waterman (crates/smithwaterman: GATK's SmithWatermanJavaAligner) ----
 *
 * Alignments identical to GATK's (fgkl reference.rs:9-203): integer affine-gap scores, ties resolved
 * in favour of the diagonal, then the insertion, then the deletion, and GATK's overhang strategies.
 * CIGAR elements are packed as in BAM: length << 4 | operation, with M = 0, I = 1, D = 2, S = 4, in
 * alternate order. `offset` is GATK's alignmentOffset. Both sequences must be non-empty
 * (FGKL_E_EMPTY_SEQUENCE); an unknown strategy is FGKL_E_INVALID_ARGUMENT. */
#define FGKL_SW_SOFTCLIP 0      /* SWOverhangStrategy codes as FgklSmithWaterman numbers them (jni/src/lib.rs:290-296) */
#define FGKL_SW_INDEL 1
#define FGKL_SW_LEADING_INDEL 2
#define FGKL_SW_IGNORE 3

/* SWParameters (crates/smithwaterman/src/lib.rs:42-66): a positive match value, negative penalties. */
typedef struct fgkl_sw_params {
  int32_t match_value;
  int32_t mismatch_penalty;
  int32_t gap_open_penalty;
  int32_t gap_extend_penalty;
} fgkl_sw_params;

/* A batch of (reference, alternate) pairs, each side concatenated with num_pairs + 1 offsets. */
typedef struct fgkl_sw_batch {
  int64_t num_pairs;
  const uint8_t* ref_bases;
  const int64_t* ref_offsets;
  const uint8_t* alt_bases;
  const int64_t* alt_offsets;
} fgkl_sw_batch;

/* The analogue of FgklSmithWaterman.alignNative (crates/jni/src/lib.rs:271-313): one pair on the
 * calling thread's engine. Writes the CIGAR string, NUL-terminated, into `cigar` (`cigar_cap` bytes,
 * FGKL_E_OUTPUT_LENGTH when short) and the offset into *offset. */
int fgkl_sw_align(const uint8_t* ref, int64_t ref_len, const uint8_t* alt, int64_t alt_len, const fgkl_sw_params* params,
                  int32_t strategy, char* cigar, int64_t cigar_cap, int32_t* offset);
/* Elements a batch's CIGAR array must hold: Σ over pairs of (reference + alternate length + 2). */
int64_t fgkl_sw_cigar_capacity(const fgkl_sw_batch* batch);
/* The batched form on a context (its device and stream): every pair in one persistent launch, the
 * costliest first. Pair k's elements start at Σ_{j<k} (ref_j + alt_j + 2) in `cigar`, counts[k] of
 * them; offsets[k] its offset. Synchronous. */
int fgkl_sw_align_batch(fgkl_context* ctx, const fgkl_sw_batch* batch, const fgkl_sw_params* params, int32_t strategy,
                        uint32_t* cigar, int64_t cigar_len, int32_t* counts, int32_t* offsets);
/* Duration (ms, CUDA events on the context's stream) of the fill-and-traceback launch of the context's
 * last fgkl_sw_align_batch call; no counterpart in the reference (measurement support). */
int fgkl_sw_last_kernel_ms(fgkl_context* ctx, float* ms);

/* ---- allocation-free form (no counterpart in the reference) ----
 *
 * The reference has no such entry: its kernels take host slices and allocate per-thread
 * workspaces. This one is for callers that must not allocate device memory per call: code whose
 * device memory is held by a pool allocator that has already reserved the free memory (a further
 * cudaMalloc fails or fragments it), and latency-bound serving loops that cannot take the
 * device-wide synchronisation cudaFree implies while other streams run.
 *
 * One region's likelihoods, every pair computed in FP64 without haplotype sharing (the value
 * Precision::Double gives, to rounding), from caller-owned arrays in the CURRENT device's memory,
 * enqueued on `stream` (a cudaStream_t, NULL = the legacy default stream) without waiting.
 * out[r * num_haplotypes + h] receives read r against haplotype h (device memory, not aliasing the
 * inputs).
 *
 * It allocates nothing: no cudaMalloc, cudaFree, pinned or library allocation. Its scratch is a
 * file-scope device array of FGKL_NOALLOC_SCRATCH_BYTES (2 MiB): a 256-byte header holding the
 * pair counter, which must start at zero and which each call zeroes with cudaMemsetAsync on
 * `stream` before its launch, then 256 bytes per resident warp (the grid is sized so they fit).
 * The first call on each device does the setup -- resolves the array's address with
 * cudaGetSymbolAddress and uploads the probability tables with synchronous copies -- so make it
 * before any stream capture.
 *
 * Calls share the one scratch array per device: two calls whose kernels overlap (different
 * streams, or threads, without ordering between them) race on it and give wrong results. Order
 * them on one stream or with events.
 *
 * Limits: max_read_len (the caller's bound on every read length) in 1..620, else
 * FGKL_E_UNSUPPORTED; num_reads x num_haplotypes at most FGKL_NOALLOC_MAX_PAIRS, else
 * FGKL_E_INVALID_ARGUMENT. The arrays are not read on the host, so a read longer than
 * max_read_len, or an empty read or haplotype, yields NaN for its pairs instead of an error. */
#define FGKL_NOALLOC_SCRATCH_BYTES (2 * 1024 * 1024)
#define FGKL_NOALLOC_MAX_READ_LEN 620
#define FGKL_NOALLOC_MAX_PAIRS 2147483647LL

typedef struct fgkl_device_region {
  int32_t num_reads;
  int32_t num_haplotypes;
  const uint8_t* bases;        /* device; reads concatenated */
  const uint8_t* quals;        /* device; same length */
  const uint8_t* ins_quals;    /* device; same length */
  const uint8_t* del_quals;    /* device; same length */
  const uint8_t* gcp;          /* device; same length */
  const int64_t* read_offsets; /* device; num_reads + 1 byte offsets */
  const uint8_t* hap_bases;    /* device; haplotypes concatenated */
  const int64_t* hap_offsets;  /* device; num_haplotypes + 1 byte offsets */
  int32_t max_read_len;        /* host-known bound on every read's length */
} fgkl_device_region;

int fgkl_pairhmm_compute_device_noalloc(const fgkl_device_region* region, double* out, void* stream);

/* ---- measurement support ---- */

/* Measured FP32 FMA throughput of `device` (TFLOP/s) with scalar FFMA and packed FP32x2 FFMA chains:
 * the denominator of the kernels' FP32 roofline. */
int fgkl_probe_fp32_tflops(int32_t device, double* scalar_tflops, double* packed_tflops, double* sm_clock_mhz);
/* Measured integer ALU throughput of `device` (Gop/s: independent chains of 32-bit XOR and signed
 * max): the denominator of the Smith-Waterman kernel's roofline. */
int fgkl_probe_int32_alu_gops(int32_t device, double* gops);

/* ---- synthetic workloads (the analogue of fgkl's crates/pairhmm/src/synthetic.rs) ---- */

typedef struct fgkl_synth fgkl_synth;
/* A benchmark workload (0-4, see synthetic.h); `regions` 0 keeps its default region count. */
fgkl_synth* fgkl_synth_config(int32_t which, uint64_t seed, int32_t regions, int32_t threads);
/* One region drawn exactly as fgkl's Region::generate (pd = 0) or PdRegion::generate (pd = 1). */
fgkl_synth* fgkl_synth_reference_region(uint64_t seed, int64_t reads, int64_t read_len, int64_t haps, int64_t hap_len,
                                        int32_t pd);
/* Points `out` into the workload; sizes = {total reads, read bases, total haplotypes, haplotype bases}. */
void fgkl_synth_view(const fgkl_synth* s, fgkl_batch* out, int64_t sizes[4]);
void fgkl_synth_free(fgkl_synth* s);

/* ---- planner diagnostics (SortedHaps::new, kernel.rs:53-81; SuffixPlan::new, plan.rs:61-89) ---- */

/* Sorted order, LCP, duplicate flags, cuts (column -1: none), sweep and node counts and the
 * SharedColumns {prefix_only, forward, backward} of one haplotype set. */
int fgkl_plan_describe(const uint8_t* hap_bases, const int32_t* hap_offsets, int32_t num_haps, int32_t share_suffixes,
                       int32_t* order, int32_t* lcp, uint8_t* dup, int32_t* cut_column, int32_t* cut_node,
                       int32_t* num_sweeps, int32_t* num_nodes, uint64_t columns[3]);
/* Per region of `batch`, the DP cells (forward + backward) a batched run computes under `config`, as
 * the planner emits them (host only, no device): the cost by which regions are balanced across
 * devices (fgkl runs regions independently, docs/design.md:37-39). `cells` has num_regions entries. */
int fgkl_plan_region_cells(const fgkl_batch* batch, const fgkl_config* config, uint64_t* cells);
/* Backward sweeps: 6 ints each (hap, resume, need, start, first write, write count) and the
 * (depth, node) writes, 2 ints each. */
int fgkl_plan_sweeps(const uint8_t* hap_bases, const int32_t* hap_offsets, int32_t num_haps, int32_t* sweeps,
                     int32_t max_sweeps, int32_t* writes, int32_t max_writes);

/* ---- PD planner diagnostics (SortedPdHaps::new, segments, MatchSet: pd_kernel.rs:61-136, :196-214,
 * :699-723) ---- */

/* Deletion state (0 normal, 1 inside a deletion, 2 after one) of each of a row's `len` columns when
 * the row starts in `start_state`; returns the state carried out of the row, or a negative code. */
int fgkl_pd_row_states(const uint8_t* flags, int32_t len, int32_t start_state, uint8_t* states);
/* Sorted order, LCP, duplicate flags and row-end states of a PD haplotype set, and its number of
 * distinct match-set codes. */
int fgkl_pd_plan_describe(const uint8_t* hap_bases, const uint8_t* hap_flags, const int32_t* hap_offsets, int32_t num_haps,
                          int32_t* order, int32_t* lcp, uint8_t* dup, uint8_t* end_state, int32_t* num_codes);
/* 1 when a PD column of base `base` and flags `flag` accepts `read_base` as a match, else 0. */
int fgkl_pd_match_accepts(uint8_t base, uint8_t flag, uint8_t read_base);

#ifdef __cplusplus
}
#endif

#endif /* FGKL_B200_H */
