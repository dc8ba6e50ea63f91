/*
 * TEST INFRASTRUCTURE — CPU oracle for C = A·B (B given explicitly, = Aᵀ in
 * every configuration here).  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only to check or time against
 * the GPU product; the product never calls it.
 *
 * It restates, in plain single-node C, the algorithm of the reference's three
 * CPU drivers (fukien/contention-aware-spgemm): per-row flop count, exclusive
 * scan, linear-probing hash symbolic phase, and the hash / ESC / hybrid
 * numeric accumulators.  Each function cites the reference lines it follows.
 * The CSR layout is the reference's csr_t (src/inc/store.h:49-56): int64 row
 * pointers and column indices, fp64 values.
 *
 * Parity is pinned: tests/test_oracle.py checks this restatement against the
 * reference itself (oracle/_ref, built from the reference's sources) and
 * against committed golden fixtures.
 */
#ifndef CAS_ORACLE_H
#define CAS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
	int64_t num_row;
	int64_t num_col;
	int64_t num_nnz;
	int64_t *row_ptrs;
	int64_t *cols;
	double *rats;
} orc_csr;

enum { ORC_HASH = 0, ORC_HSERSC = 1, ORC_HYBACC = 2 };

/* NEXT_POW_2 of src/inc/utils.h:92, computed exactly on integers. */
int64_t orc_next_pow2(int64_t x);

/* row_flp[i] = sum over k in A_i of |B_k| (flp_populate, src/mm/mm_utils.c:1063-1125). */
void orc_flp_populate(const orc_csr *A, const orc_csr *B, int64_t *row_flp);

/* out[0] = 0, out[i+1] = out[i] + in[i] for i < n-1 (scan, src/mm/mm_utils.c:903-911). */
void orc_scan(int64_t *out, const int64_t *in, int64_t n);

/* Sum of row_flp (get_intprod, src/mm/mm_utils.c:981-1055). */
int64_t orc_intprod(const orc_csr *A, const orc_csr *B);

/* Exact number of distinct columns per row of A·B by linear probing
 * (pthread_ams_hash_symb_dnr, src/ams/ams_utils.c:1630-1699). */
void orc_hash_symb(const orc_csr *A, const orc_csr *B, const int64_t *row_flp, int64_t *row_nz);

/* Stable LSD byte radix sort of (key, val) pairs with the early-outs of
 * radix_sort_keyval_toggling_unrolling (src/mm/mm_utils.c:1273-1375).
 * keys/vals are sorted in place; aux_k/aux_v are scratch of length n. */
void orc_radix_sort_kv(int64_t *keys, double *vals, int64_t *aux_k, double *aux_v, int64_t n);

/* Full pipeline: flop count, hash symbolic, scan, numeric with the chosen
 * accumulator (ams_hash_numc_krnl src/ams/ams_utils.c:168-328,
 * ams_hsersc_numc_krnl :335-475, ams_hybacc_numc_krnl :1080-1155 with the
 * per-row choice cf < acc_thres -> ESC).  C's arrays are malloc'd; rows are
 * left in the order the accumulator emits them (hash: slot order) unless
 * sort_rows != 0.  Returns the total intermediate products. */
int64_t orc_spgemm(const orc_csr *A, const orc_csr *B, orc_csr *C, int algo,
	double acc_thres, int sort_rows);

/* Sort the entries of every row by column (the canonical form used for
 * parity: the hash accumulator emits rows in slot order). */
void orc_sort_rows(orc_csr *C);

/* Morsel packing of pack_ams_pack (src/ams/ams_utils.c:1410-1596, default
 * build without AMS_MAXFLP): morsel j covers rows
 * [bounds[j], bounds[j+1]) where bounds[j+1] = lower_bound(ps_weight,
 * morsel*(j+1)) and the last bound is num_row; cf[j] = (ps_flp[e]-ps_flp[s]) /
 * (ps_weight[e]-ps_weight[s]) (0 for empty morsels), maxflp[j] = max row_flp.
 * order[] is the morsel index sorted by (cf, index) ascending
 * (compare_keyvals_3, src/mm/mm_utils.c:57-65).  Arrays must hold
 * total = ps_weight[num_row] / morsel entries (bounds: total+1).
 * Returns total; *low_head = number of empty morsels; *high_tail =
 * (total - low_head) * prt + low_head (src/ams/ams_utils.c:1571-1573). */
int64_t orc_pack_morsels(int64_t num_row, const int64_t *ps_weight, const int64_t *row_flp,
	const int64_t *ps_flp, int64_t morsel, double prt, int64_t *bounds, double *cf,
	int64_t *maxflp, int64_t *order, int64_t *low_head, int64_t *high_tail);

/* Row digests of C in the form of the casgemm ABI's cas_csr_digest (no
 * counterpart in the reference, whose IN_VERIFY build prints only nnz, the
 * column sum and the value sum, src/ams_hashspgemm.c:307-318):
 *   h(c, k, v) = mix64(c * 0x9E3779B97F4A7C15 + k) ^ mix64(bits(v) + 0x632BE59BD9B4E019)
 *   row_digests[r] = sum over the row's entries in stored order, k = 0, 1, ...
 * with mix64 the SplitMix64 finaliser (Steele, Lea, Flood 2014), bits(v) the
 * fp64 bit pattern, sums modulo 2^64.  Rows should be sorted first
 * (orc_sort_rows) for a canonical digest.  Returns the product digest
 * sum over r of mix64(row_digests[r] + r + row_offset). */
uint64_t orc_row_digests(const orc_csr *C, int64_t row_offset, uint64_t *row_digests);

void orc_free(orc_csr *C);

#ifdef __cplusplus
}
#endif
#endif
