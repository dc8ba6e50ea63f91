/*
 * casgemm data layer: seeded synthetic inputs, MatrixMarket I/O in the
 * reference's format, and host-side CSR helpers.
 *
 * Matrices are CSR with int64 row pointers and int32 column indices.  Every
 * generator is a pure function of its parameters and seed (counter-based
 * random numbers), and independent of the number of host threads.
 *
 * Replaces the reference's dataset preparation: PaRMAT (PaRMAT/src/, unseeded)
 * followed by rmat_ones (src/rmat_ones.c:6-37, src/mm/mm_utils.c:759-862), and
 * the MatrixMarket loader raw2csr/mtx2trpl/trpl2csr (src/mm/mm_utils.c:451-692,
 * src/mm/mm_utils.c:730).
 */
#ifndef CASGEMM_DATA_H
#define CASGEMM_DATA_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Undirected R-MAT graph on 2^scale vertices with exactly edge_factor*2^scale
 * distinct loop-free edges, symmetrised: row_ptrs[2^scale + 1], cols[2 *
 * edge_factor * 2^scale] (caller-allocated), rows sorted by column.  Each
 * candidate edge draws its quadrant at every level with probabilities
 * a, b, c, 1-a-b-c; self-loops are dropped, and of repeated edges the first
 * occurrence in candidate order is kept until the target count is reached.
 * Returns 0, or -1 on bad parameters / allocation failure. */
int cas_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
	int64_t *row_ptrs, int32_t *cols);

/* Rows of a Zipf bipartite matrix: deg(r) = max(1, round(amax * ((1+q)/(r+q))^row_s))
 * for r = 1..num_row, with q solved so that the degrees sum to target_nnz
 * (within rounding).  Writes the degrees in generated-row order to deg[] and
 * returns q, or a negative value on failure. */
double cas_zipf_row_degrees(int64_t num_row, int64_t amax, double row_s, int64_t target_nnz,
	int64_t *deg);

/* Zipf bipartite matrix: row degrees from cas_zipf_row_degrees (rows then
 * shuffled by the seed), each row holding deg distinct columns drawn with
 * p_k proportional to (k + col_q)^-col_s, k = 1..num_col.  Two-phase: call with
 * cols == NULL to get nnz (returned) and row_ptrs filled; then with cols of
 * that length.  Returns nnz, or -1 on failure. */
int64_t cas_gen_zipf(int64_t num_row, int64_t num_col, int64_t amax, double row_s,
	int64_t target_nnz, double col_s, double col_q, uint64_t seed,
	int64_t *row_ptrs, int32_t *cols);

/* Uniform integer values in [lo, hi] for nnz entries (seeded). */
void cas_gen_int_values(int64_t nnz, int32_t lo, int32_t hi, uint64_t seed, int32_t *vals);

/* Host CSR transpose: B = A^T with B rows sorted by column.  vals may be NULL
 * (pattern only); val_bytes is 4 or 8.  Caller allocates B (num_col+1 row
 * pointers, nnz cols/vals). */
int cas_csr_transpose_host(int64_t num_row, int64_t num_col, const int64_t *row_ptrs,
	const int32_t *cols, const void *vals, int val_bytes,
	int64_t *t_row_ptrs, int32_t *t_cols, void *t_vals);

/* Intermediate products of A*B: sum over nnz of A of |B_col| (the
 * reference's flop_cnt, get_intprod src/mm/mm_utils.c:981-1055). */
int64_t cas_intprod_host(int64_t num_row, const int64_t *a_row_ptrs, const int32_t *a_cols,
	const int64_t *b_row_ptrs);

/* MatrixMarket coordinate file -> CSR with the reference loader's semantics
 * (mtx2trpl, src/mm/mm_utils.c:451-607): '%' lines skipped, "symmetric" in a
 * comment mirrors every off-diagonal entry, explicit zeros dropped, every
 * value forced to 1.0, 1-based -> 0-based, entries sorted by (row, col),
 * duplicates kept.  Two-phase like cas_gen_zipf: cols == NULL returns nnz and
 * the shape; the second call fills row_ptrs/cols/vals.  Returns nnz or -1. */
int64_t cas_mtx_read(const char *path, int64_t *num_row, int64_t *num_col,
	int64_t *row_ptrs, int32_t *cols, double *vals);

/* CSR -> MatrixMarket in the format trpl2mtx writes (src/mm/mm_utils.c:611-647):
 * symmetric != 0 writes the "symmetric" header and only entries with
 * row <= col; values are written as 1.000000.  Returns 0 or -1. */
int cas_mtx_write(const char *path, int64_t num_row, int64_t num_col, const int64_t *row_ptrs,
	const int32_t *cols, int symmetric);

/* Binary CSR cache, so a dataset is parsed from MatrixMarket once: the
 * bytes "CASCSR1" and a NUL, then num_row, num_col and nnz as int64, then
 * row_ptrs (num_row + 1 int64), cols (nnz int32) and vals (nnz double), all
 * little-endian.  No counterpart in the reference, which parses the .mtx
 * files on every run (raw2csr, src/mm/mm_utils.c:451-692).  Write returns 0
 * or -1.  Read is two-phase like cas_mtx_read (cols == NULL returns nnz and
 * the shape) and returns nnz, or -1 on a missing or malformed file. */
int cas_csr_write_bin(const char *path, int64_t num_row, int64_t num_col, const int64_t *row_ptrs,
	const int32_t *cols, const double *vals);
int64_t cas_csr_read_bin(const char *path, int64_t *num_row, int64_t *num_col, int64_t *row_ptrs,
	int32_t *cols, double *vals);

#ifdef __cplusplus
}
#endif
#endif
