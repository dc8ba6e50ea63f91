/*
 * casgemm — C = A·B sparse-sparse product on one NVIDIA B200 (sm_100a), the
 * drop-in for the CPU SpGEMM of fukien/contention-aware-spgemm (C = A·Aᵀ with
 * B = Aᵀ read as its own CSR, as the reference's drivers do).
 *
 * Plain C ABI: pointers, sizes, status codes; no C++ or torch types.
 * Every function returns a cas_status; on failure cas_last_error() describes
 * it.  A context is bound to one device and one CUDA stream and is not
 * re-entrant (the reference is not either: it keeps process-global state,
 * src/ams/ams_utils.c:29-33); use one context per host thread.
 *
 * Output: every row of C has its columns sorted ascending, and each value is
 * the sum of its products.  The reference's hash accumulator leaves rows in
 * hash-slot order (src/ams/ams_utils.c:301-309); sorted rows are the same set
 * of (row, col, value) entries.
 */
#ifndef CASGEMM_H
#define CASGEMM_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
	CAS_OK = 0,
	CAS_ERR_BAD_INPUT = 1,   /* shapes, pointers or index widths are invalid */
	CAS_ERR_OOM = 2,         /* device or host allocation failed */
	CAS_ERR_CUDA = 3,        /* a CUDA call failed */
	CAS_ERR_DEVICE = 4,      /* a device-side guard fired (see cas_last_error) */
	CAS_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
	CAS_ERR_ABORTED = 6,     /* cancelled by the caller */
	CAS_ERR_REJECTED = 7     /* a request that can never fit the memory budget */
} cas_status;

/* The three accumulators of the reference's drivers. */
typedef enum {
	CAS_ACC_HASH = 0,    /* ams_hashspgemm   (ams_hash_numc,   src/ams/ams_utils.c:608)  */
	CAS_ACC_HSERSC = 1,  /* ams_hserscspgemm (ams_hsersc_numc, src/ams/ams_utils.c:781)  */
	CAS_ACC_HYBACC = 2   /* ams_hybaccspgemm (ams_hybacc_numc, src/ams/ams_utils.c:1159) */
} cas_accum;

/* Value arithmetic. */
typedef enum {
	CAS_VAL_F64 = 0,     /* fp64 in, fp64 out (the reference's my_rat_t, src/inc/store.h:20) */
	CAS_VAL_I32 = 1      /* int32 in, int64 out (exact integer accumulation) */
} cas_valtype;

/* CSR matrix.  Layout-compatible with the reference's csr_t
 * (src/inc/store.h:49-56) when col_bytes == 8, val_type == CAS_VAL_F64 and
 * on_device == 0: the first six fields line up. */
typedef struct {
	int64_t num_row;
	int64_t num_col;
	int64_t num_nnz;
	int64_t *row_ptrs;   /* num_row + 1 entries */
	void *cols;          /* int32 (col_bytes 4) or int64 (col_bytes 8) column indices */
	void *rats;          /* values: double, or int32 input / int64 output for CAS_VAL_I32 */
	int32_t col_bytes;   /* 4 or 8; device matrices use 4 */
	int32_t val_type;    /* cas_valtype */
	int32_t on_device;   /* 1: pointers are device memory of the context's device */
	int32_t owned;       /* set by the library when it allocated the arrays (2: host arrays from the
	                        context's block cache); see cas_csr_free */
} cas_csr;

/* Phase times in seconds, the reference's runtime_t (src/mm/mm_utils.h:48-54);
 * measured with CUDA events on the context's stream. */
typedef struct {
	double init_time;
	double symb_time;
	double mgmt_time;
	double numc_time;
	double total_time;
} cas_runtime;

#define CAS_SYMB_BINS 9
#define CAS_NUMC_BINS 13

/* Counters of the last cas_spgemm call. */
typedef struct {
	int64_t flop;                          /* intermediate products (flop_cnt, get_intprod) */
	int64_t max_row_flp;                   /* largest row product count */
	int64_t nnz_c;
	int64_t symb_bin_rows[CAS_SYMB_BINS];  /* rows per symbolic bin */
	int64_t numc_bin_rows[CAS_NUMC_BINS];  /* rows per numeric bin */
	int64_t kernel_launches;               /* kernels launched by the library since cas_create */
	double h2d_bytes;                      /* host->device bytes copied by the call */
	double d2h_bytes;                      /* device->host bytes copied by the call */
	/* with cas_set_profiling(ctx, 1): device time of each bin's kernel (ms,
	 * CUDA events on the stream it ran on) and, for the numeric bins, the
	 * algorithmic bytes of its rows: 12*nnz(A rows) + 12*products +
	 * 12*nnz(C rows) + 16*rows for fp64 (int32 in / int64 out: 8/8/12/16). */
	double symb_bin_ms[CAS_SYMB_BINS];
	double numc_bin_ms[CAS_NUMC_BINS];
	double numc_bin_bytes[CAS_NUMC_BINS];
	int64_t numc_bin_flop[CAS_NUMC_BINS];
	/* rows the bucketed ESC kernel handed to the radix-sort ESC kernel (their
	 * columns crowd into a narrow range), and that kernel's time (profiling) */
	int64_t esc_overflow_rows;
	double esc_overflow_ms;
	/* rows of the fused ESC kernel (no symbolic pass; see cas_set_fusion),
	 * their products and algorithmic bytes (as above), its time (profiling) */
	int64_t fused_rows;
	int64_t fused_flop;
	double fused_bytes;
	double fused_ms;
	/* of d2h_bytes, those copied by DMA straight into host blocks the
	 * context has registered (blocks it kept from earlier outputs) */
	double d2h_direct_bytes;
	/* dense rows split across thread blocks (cas_tuning.heavy_split) */
	int64_t split_rows;
	/* row blocks the call computed C in (cas_tuning.out_blocks; 1 for a C
	 * in device memory) */
	int64_t out_blocks;
	/* nnz(C) of the rows of each numeric bin (the fused rows are not in them) */
	int64_t numc_bin_nnz[CAS_NUMC_BINS];
} cas_stats;

typedef struct cas_ctx cas_ctx;

/* Context on `device`; the stream is a new non-blocking stream. */
cas_status cas_create(int device, cas_ctx **out);
void cas_destroy(cas_ctx *ctx);
/* Use an existing cudaStream_t (passed as void*); NULL restores the context's own. */
cas_status cas_set_stream(cas_ctx *ctx, void *stream);
/* AMS_ACC_THRES of the hybrid accumulator (cmake/Options.cmake:142-146):
 * rows with products/nnz below it take ESC.  Default 2.0, the R-MAT run
 * script's value for ams_hybaccspgemm (scripts/ams_rmat_run.sh:33). */
cas_status cas_set_acc_thres(cas_ctx *ctx, double thres);
const char *cas_last_error(const cas_ctx *ctx);
/* 1 (default): in cas_spgemm with the ESC or hybrid accumulator, rows of
 * 2049..5120 products (the lower bound is cas_tuning.fused_min_products)
 * skip the symbolic pass: one kernel counts, sorts and
 * places each of them, finding its offset in C from the rows before it, and
 * C is allocated by the bound min(products, columns) for those rows
 * (C->num_nnz is exact; the arrays may be longer).  0: every row has a
 * symbolic pass, as in the reference's drivers.  The output is the same. */
cas_status cas_set_fusion(cas_ctx *ctx, int on);

/* Routing of rows to kernels, all of it in one place (the defaults in
 * brackets).  The output never depends on it, only the speed: the
 * project's autotuner (casgemm.Autotuner) times candidate settings per
 * degree-distribution class of the inputs and keeps the fastest.
 * No counterpart in the reference beyond AMS_ACC_THRES, whose
 * thresholds are compile-time macros (CMakeLists.txt:57-65). */
typedef struct {
	double acc_thres;            /* AMS_ACC_THRES of the hybrid accumulator [2.0] */
	int32_t fusion;              /* fused ESC rows, as cas_set_fusion [1] */
	int32_t fused_min_products;  /* fused rows have more products than this, up to 5120 [2048] */
	int32_t esc_max_products;    /* ESC rows have at most this many products, <= 8192 [8192] */
	int32_t hash_max_nnz;        /* hash rows have at most this many distinct columns, <= 4096 [4096];
	                                larger rows take the dense kernels */
	int32_t esc_form;            /* bucketed ESC kernel of the fused rows and of ESC rows over 4096
	                                products: 1 keeps column, product index and place per product in
	                                shared memory, 4 rows per SM; 2 [the default] is form 1 with each thread's
	                                columns held in registers between its histogram and scatter
	                                passes (B's columns read once) and, for rows whose B rows average
	                                32 products or more, a warp per B row in the value pass (rows of
	                                up to 6144 products; larger ones take form 1); 0 keeps column and
	                                value, 3 rows per SM */
	int32_t heavy_split;         /* 1: dense rows of 2^17 products or more are split across thread blocks
	                                by A-entry ranges, heaviest row first, adding into C by atomics that
	                                stay in L2 [1]; 0: one block per dense row */
	int32_t bin_order;           /* 1: the numeric bins of contended rows (dense, hash) launch first on
	                                the auxiliary streams, the ESC bins after them [1]; 0: the two
	                                kinds interleaved, so they run side by side, as the reference's
	                                high- and low-contention thread groups claim morsels from the two
	                                ends of its cf-sorted queue (src/ams/ams_utils.c:190-216) */
	int32_t out_blocks;          /* C returned in host memory (int32 columns) is computed in this many
	                                row blocks of about equal A entries, each copied out while the next
	                                is computed, into host arrays sized by sum over rows of
	                                min(products, num_col); 0: one block under 1 GiB of C, else one per
	                                2 GiB, at least 2 and at most 64 [0]; 1: one block, host arrays
	                                sized by the symbolic counts; at most 64 */
} cas_tuning;
cas_status cas_set_tuning(cas_ctx *ctx, const cas_tuning *t);
cas_status cas_get_tuning(const cas_ctx *ctx, cas_tuning *t);
/* 1: run the bins one after another on the context's stream and time every
 * bin kernel with CUDA events (cas_stats.*_bin_ms); 0 (default): bins run
 * concurrently on auxiliary streams. */
cas_status cas_set_profiling(cas_ctx *ctx, int on);
cas_status cas_get_stats(const cas_ctx *ctx, cas_stats *out);

/* ---- the reference's phase functions, on device CSR (col_bytes 4) ------ */

/* row_flp[i] = sum over A_i of |B_k| into device memory (m entries).
 * Replaces flp_populate (src/mm/mm_utils.c:1089-1125). */
cas_status cas_flp_populate(cas_ctx *ctx, const cas_csr *A, const cas_csr *B, int64_t *d_row_flp);

/* d_out[0] = 0, d_out[i+1] = d_out[i] + d_in[i] for i < n-1 (device arrays).
 * Replaces scan (src/mm/mm_utils.c:903-957). */
cas_status cas_scan(cas_ctx *ctx, int64_t *d_out, const int64_t *d_in, int64_t n);

/* Exact distinct-column count of every row of A·B into d_row_nz (m entries).
 * Replaces ams_hash_symb_dnr (src/ams/ams_utils.c:1701-1752) and
 * ams_hash_symb (:483-602).  d_row_flp (from cas_flp_populate) is taken for
 * the reference's signature and may be NULL: this call and the numeric calls
 * below recompute the row products in the same pass that bins the rows by
 * kernel, which reads A and B's row pointers once, so the caller's array is
 * neither read nor written. */
cas_status cas_hash_symb(cas_ctx *ctx, const cas_csr *A, const cas_csr *B, const int64_t *d_row_flp,
	int64_t *d_row_nz);

/* Numeric phase into a caller-allocated device C whose row_ptrs are the scan
 * of the symbolic counts (C->num_nnz entries of cols/rats); d_row_flp as in
 * cas_hash_symb.  Rows of more than 4096 distinct columns take the dense
 * kernel, which builds its column bitmaps itself here (cas_spgemm keeps them
 * from its symbolic pass).
 * Replace ams_hash_numc (src/ams/ams_utils.c:608-774), ams_hsersc_numc
 * (:781-949) and ams_hybacc_numc (:1159-1338). */
cas_status cas_hash_numc(cas_ctx *ctx, const cas_csr *A, const cas_csr *B, const int64_t *d_row_flp,
	cas_csr *C);
cas_status cas_hsersc_numc(cas_ctx *ctx, const cas_csr *A, const cas_csr *B, const int64_t *d_row_flp,
	cas_csr *C);
cas_status cas_hybacc_numc(cas_ctx *ctx, const cas_csr *A, const cas_csr *B, const int64_t *d_row_flp,
	cas_csr *C);

/* ---- whole product --------------------------------------------------- */

/* C = A·B with the given accumulator: the four phases of the drivers'
 * hashspgemm / hserscspgemm / hybaccspgemm (src/ams_hashspgemm.c:36-205,
 * src/ams_hserscspgemm.c:36-210, src/ams_hybaccspgemm.c:36-215).
 * A and B may be host (either column width) or device (col_bytes 4) CSR.
 * C is allocated by the library: on the device when C->on_device is 1 on
 * entry (col_bytes 4), else in host memory with C->col_bytes (4 or 8) columns.
 * C->val_type is CAS_VAL_F64 for fp64 inputs and CAS_VAL_I32 (int64 values)
 * for int32 inputs.  Release C with cas_csr_free.  rt may be NULL. */
cas_status cas_spgemm(cas_ctx *ctx, cas_accum accum, const cas_csr *A, const cas_csr *B, cas_csr *C,
	cas_runtime *rt);

/* Frees arrays the library allocated (owned != 0) and zeroes the struct.
 * Host arrays of a C from cas_spgemm (owned 2) go back to the context that
 * made them, which keeps up to 60% of physical memory of such blocks, pages
 * resident, for later outputs (so repeated products into host memory skip
 * the page faults); they are released at cas_destroy.  Passing another
 * context or NULL frees them at once, after releasing them from the context
 * that made them (and unregistering them from CUDA where it had registered
 * them); this is safe from any thread. */
cas_status cas_csr_free(cas_ctx *ctx, cas_csr *C);

/* ---- the second input: B = Aᵀ on the device -------------------------------
 *
 * B = Aᵀ made on the device from A, so a caller with A alone needs no
 * transposed file.  Replaces the reference's trpl_transpose
 * (src/mm/mm_utils.c:742-754), which swaps every triple's row and column and
 * sorts the triples by (row, column) before txt_transpose (:851-862) writes
 * them to <dataset>.trs.mtx for the drivers to read.  A is a host CSR (int32
 * or int64 columns) or a device CSR (col_bytes 4), checked on the device
 * (CAS_ERR_BAD_INPUT for row pointers or columns out of range).  B is
 * allocated by the library: on the device when B->on_device is 1 on entry,
 * else in host memory; col_bytes 4, A's value type; release it with
 * cas_csr_free.  Rows of B are sorted by column, and duplicate (row, column)
 * entries of A keep their order, so B equals the host's stable
 * counting-sort transpose entry for entry. */
cas_status cas_csr_transpose(cas_ctx *ctx, const cas_csr *A, cas_csr *B);

/* ---- digests of a product ------------------------------------------------
 *
 * A 64-bit digest of a CSR C that depends on every row's entries in order,
 * so two products agree bit for bit if their digests do (up to collisions):
 *   h(c, k, v) = mix64(c * 0x9E3779B97F4A7C15 + k) ^ mix64(bits(v) + 0x632BE59BD9B4E019)
 *   row_digest[r] = sum over the row's entries, k = 0, 1, ... of h(col_k, k, val_k)
 *   digest = sum over rows r of mix64(row_digest[r] + r)
 * all sums modulo 2^64; mix64 is the SplitMix64 finaliser (Steele, Lea,
 * Flood 2014); bits(v) is the fp64 bit pattern, or the int64 value for
 * CAS_VAL_I32 outputs.  No counterpart in the reference, whose IN_VERIFY
 * build prints nnz, the sum of columns and the sum of values
 * (src/ams_hashspgemm.c:307-318). */
cas_status cas_csr_digest(cas_ctx *ctx, const cas_csr *C, uint64_t *digest, uint64_t *row_digests);

/* ---- batches of independent products -------------------------------------
 *
 * No counterpart in the reference, which runs one product per process.  A
 * batch runs many independent products C_j = A_j * B_j of uneven sizes on
 * one device.  Outputs are not kept: each job reports its product count,
 * nnz(C_j), the digest above, and per-row digests when row_digests is set
 * (a host array of A_j.num_row entries). */
typedef struct {
	cas_csr A, B;            /* inputs: host or device (col_bytes 4), one value type per batch */
	uint64_t *row_digests;   /* optional host output, A.num_row entries */
	int64_t flop;            /* out: intermediate products */
	int64_t nnz_c;           /* out */
	uint64_t digest;         /* out */
	int32_t status;          /* out: cas_status of the job */
} cas_job;

typedef enum {
	/* All jobs as one block-diagonal product diag(A_j) * diag(B_j): the
	 * inputs are packed into one device CSR pair (columns shifted per job), the
	 * rows run in waves that fit wave_budget bytes of output by the bound
	 * 12 * min(products, columns) per row, and each wave's bins launch once
	 * over the rows of every job in it. */
	CAS_BATCH_WAVES = 0,
	/* One cas_spgemm per job, in order: the same kernels, launched per job. */
	CAS_BATCH_PER_CALL = 1,
	/* The jobs as in PER_CALL on 4 host threads, each with a context of its
	 * own (created on first use and kept by the calling context): the
	 * threads claim jobs from a shared counter, largest first by the estimate
	 * nnz(A) * nnz(B) / rows(B), so one job's host waits overlap the others'
	 * kernels and small jobs' kernels run side by side.  Each worker sizes its
	 * optional scratch by a quarter of the free device memory, and a job that
	 * still runs out of device memory beside the others is run again after
	 * them, alone, on the calling context.  stats->seconds runs
	 * from the batch's start on the calling context's stream to the last
	 * worker's last kernel; kernel_launches counts the workers' launches. */
	CAS_BATCH_CONCURRENT = 2
} cas_batch_mode;

typedef struct {
	double seconds;          /* device time from the first copy to the last digest (CUDA events) */
	int64_t waves;           /* products run (waves, or jobs for PER_CALL) */
	int64_t jobs_ok;
	int64_t flop;            /* sum over jobs */
	int64_t nnz_c;           /* sum over jobs */
	int64_t kernel_launches; /* library kernels launched by the batch */
	double h2d_bytes;
	double max_wave_bound;   /* largest wave's output bound, bytes */
} cas_batch_stats;

/* Runs the batch; wave_budget <= 0 means 32 GiB.  Returns CAS_OK when every
 * job succeeded, else the first failure (each job's status says which). */
cas_status cas_batch_run(cas_ctx *ctx, cas_accum accum, cas_job *jobs, int64_t n, cas_batch_mode mode,
	double wave_budget, cas_batch_stats *stats);

/* ---- serving: a request loop with continuous batching --------------------
 *
 * No counterpart in the reference.  A server owns `slots` worker threads,
 * each with its own context and streams on one device.  cas_serve_submit
 * queues a request and returns at once.  Requests are admitted in arrival
 * order, each when a slot is free and its device-memory bound fits the
 * budget beside the requests already running:
 *   bound = 12 * sum over rows of min(row products, B.num_col) + 40 * (m + 1)
 *           + the device copies of A and B
 * (C's entries and row pointers, A's row pointers and the pipeline's per-row
 * scratch), computed at submission from the row products.  Admitted requests
 * run concurrently on the device, and later arrivals join as slots and
 * memory free up.  A request whose bound exceeds the whole budget runs in row
 * chunks that each fit.  Inputs are CSRs with col_bytes 4, both on the host
 * or both resident on the server's device (on_device 1): a caller that
 * serves the same matrices again and again uploads each once and submits
 * the device copies, so no request copies its operands.  For resident
 * operands the bound leaves out A's and B's copies (they are the caller's
 * memory), and submission computes the row products on the device and checks
 * the structure there (row pointers from 0 to nnz, columns inside B;
 * CAS_ERR_BAD_INPUT otherwise).  The server reads a request's A and B until
 * it completes, so the caller keeps those arrays alive and unchanged until
 * then.  Times are seconds on the server's monotonic clock
 * (cas_serve_clock). */
typedef struct cas_server cas_server;

typedef struct {
	int32_t slots;              /* requests in flight at once (default 4) */
	int32_t accum;              /* cas_accum (default CAS_ACC_HASH = 0; set CAS_ACC_HYBACC explicitly) */
	double mem_budget;          /* device bytes for admitted requests (<= 0: 60e9) */
	int32_t keep_output;        /* 1: C returned in host memory (cas_result.C) */
	int32_t dry_run;            /* 1: no device work; a request takes dry_run_ns_per_byte * bound ns
	                               (tests of the scheduler on machines without a GPU) */
	double dry_run_ns_per_byte;
} cas_server_opts;

typedef struct {
	int32_t status;             /* cas_status of the request */
	int32_t chunks;             /* row chunks it ran in (1 unless its bound exceeded the budget) */
	int64_t flop;
	int64_t nnz_c;
	uint64_t digest;            /* cas_csr_digest of C */
	double bound;               /* device bytes reserved while it ran */
	double t_submit, t_admit, t_done;
	cas_csr C;                  /* keep_output: host C, freed with cas_csr_free(NULL, &C) */
} cas_result;

typedef struct {
	int64_t submitted, completed, failed, chunked;
	int32_t max_inflight;       /* most requests running at once */
	double max_inflight_bytes;  /* largest sum of reserved bounds at once */
} cas_server_stats;

cas_status cas_serve_create(int device, const cas_server_opts *opts, cas_server **out);
/* Queues C = A * B; *id names the request. */
cas_status cas_serve_submit(cas_server *srv, const cas_csr *A, const cas_csr *B, int64_t *id);
/* CAS_OK with *out filled once request `id` completed (the id is then
 * released); CAS_ERR_TIMEOUT while it has not.  cas_serve_wait blocks up to
 * timeout_s seconds (< 0: without limit). */
cas_status cas_serve_poll(cas_server *srv, int64_t id, cas_result *out);
cas_status cas_serve_wait(cas_server *srv, int64_t id, double timeout_s, cas_result *out);
cas_status cas_serve_stats(cas_server *srv, cas_server_stats *out);
double cas_serve_clock(const cas_server *srv);
/* Completes every queued request, then stops the workers. */
void cas_serve_destroy(cas_server *srv);

/* ---- scan that allocates nothing ---------------------------------------- */

/* The exclusive scan of cas_scan (d_out[0] = 0, d_out[i+1] = d_out[i] +
 * d_in[i], device arrays of the current device) for callers that must not
 * allocate device memory: a process whose device memory is owned and
 * budgeted by another framework's pool, or a latency-sensitive loop that
 * cannot afford the synchronisation a cudaMalloc/cudaFree may bring.  It
 * needs no context and calls no allocator: its scratch is a fixed 128 KiB
 * array in device memory that every device loading the library keeps until
 * the process exits.
 *   - n may be at most 67,108,864 (16,384 tiles of 4,096); larger n returns
 *     CAS_ERR_REJECTED without touching memory.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress); make that first call before any stream capture.
 *   - The call is asynchronous on `stream` (a cudaStream_t as void*, NULL for
 *     the default stream); synchronise before reading d_out.
 *   - All calls share the one array: calls that may overlap on the GPU must
 *     be serialised by the caller.
 *   - The array's address is looked up once per device and kept, so the
 *     function must not be used after cudaDeviceReset (or any other teardown
 *     of the device's primary context) in the same process.
 *   - A CUDA error already pending on the calling thread makes the call
 *     return CAS_ERR_CUDA without launching, and stays pending for the
 *     caller; an error of the call's own launches is read (cleared) and
 *     reported as CAS_ERR_CUDA.
 * No counterpart in the reference: its scan (src/mm/mm_utils.c:903) runs on
 * the host and allocates nothing on a device to begin with. */
cas_status cas_scan_noalloc(int64_t *d_out, const int64_t *d_in, int64_t n, void *stream);

#ifdef __cplusplus
}
#endif
#endif
