/*
 * TEST INFRASTRUCTURE — CPU oracle (see cas_oracle.h).  Restates the
 * reference's algorithm; rows are independent, so the loops over rows run
 * under OpenMP with per-thread scratch and give the same result for any
 * thread count.
 */
#include "cas_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

/* HASH_CONSTANT of the run-script build (cmake/Options.cmake:82-90,
 * scripts/ams_run_common.sh:32). */
#define ORC_HASH_CONSTANT 2654435761ULL

int64_t orc_next_pow2(int64_t x) {
	int64_t p = 1;
	while (p < x) {
		p <<= 1;
	}
	return p;
}

/* hash = (key * HASH_CONSTANT) & (size - 1): src/ams/ams_utils.c:1672.
 * Computed in uint64, which has the same low bits as the reference's int64
 * product. */
static inline int64_t orc_hash(int64_t key, int64_t size) {
	return (int64_t) (((uint64_t) key * ORC_HASH_CONSTANT) & (uint64_t) (size - 1));
}

void orc_flp_populate(const orc_csr *A, const orc_csr *B, int64_t *row_flp) {
	#pragma omp parallel for schedule(dynamic, 256)
	for (int64_t i = 0; i < A->num_row; i++) {
		int64_t flp = 0;
		for (int64_t j = A->row_ptrs[i]; j < A->row_ptrs[i + 1]; j++) {
			int64_t k = A->cols[j];
			flp += B->row_ptrs[k + 1] - B->row_ptrs[k];
		}
		row_flp[i] = flp;
	}
}

void orc_scan(int64_t *out, const int64_t *in, int64_t n) {
	if (n <= 0) {
		return;
	}
	out[0] = 0;
	for (int64_t i = 0; i < n - 1; i++) {
		out[i + 1] = out[i] + in[i];
	}
}

int64_t orc_intprod(const orc_csr *A, const orc_csr *B) {
	int64_t total = 0;
	#pragma omp parallel for reduction(+:total) schedule(dynamic, 256)
	for (int64_t i = 0; i < A->num_row; i++) {
		for (int64_t j = A->row_ptrs[i]; j < A->row_ptrs[i + 1]; j++) {
			int64_t k = A->cols[j];
			total += B->row_ptrs[k + 1] - B->row_ptrs[k];
		}
	}
	return total;
}

/* Table size of one row: NEXT_POW_2(min(row_flp, num_col))
 * (src/ams/ams_utils.c:1651-1655, hybacc variant :961-962). */
static inline int64_t orc_table_size(int64_t row_flp, int64_t num_col) {
	int64_t s = row_flp > num_col ? num_col : row_flp;
	return orc_next_pow2(s);
}

void orc_hash_symb(const orc_csr *A, const orc_csr *B, const int64_t *row_flp, int64_t *row_nz) {
	int64_t cap = orc_next_pow2(B->num_col > 0 ? B->num_col : 1);
	#pragma omp parallel
	{
		int64_t *check = (int64_t *) malloc(sizeof(int64_t) * cap);
		#pragma omp for schedule(dynamic, 256)
		for (int64_t i = 0; i < A->num_row; i++) {
			int64_t nz = 0;
			if (row_flp[i] > 0) {
				int64_t size = orc_table_size(row_flp[i], B->num_col);
				memset(check, -1, sizeof(int64_t) * size);
				for (int64_t ja = A->row_ptrs[i]; ja < A->row_ptrs[i + 1]; ja++) {
					int64_t k = A->cols[ja];
					for (int64_t jb = B->row_ptrs[k]; jb < B->row_ptrs[k + 1]; jb++) {
						int64_t key = B->cols[jb];
						int64_t h = orc_hash(key, size);
						for (;;) {
							if (check[h] == key) {
								break;
							} else if (check[h] == -1) {
								check[h] = key;
								nz++;
								break;
							}
							h = (h + 1) & (size - 1);
						}
					}
				}
			}
			row_nz[i] = nz;
		}
		free(check);
	}
}

void orc_radix_sort_kv(int64_t *keys, double *vals, int64_t *aux_k, double *aux_v, int64_t n) {
	if (n < 2) {
		return;
	}
	/* early-out when all keys are equal: src/mm/mm_utils.c:1281-1290 */
	int same = 1;
	for (int64_t i = 1; i < n; i++) {
		if (keys[i] != keys[0]) {
			same = 0;
			break;
		}
	}
	if (same) {
		return;
	}
	/* passes = bytes of the maximum key: src/mm/mm_utils.c:1296-1315 */
	int64_t max_key = 0;
	for (int64_t i = 0; i < n; i++) {
		if (keys[i] > max_key) {
			max_key = keys[i];
		}
	}
	int passes = 0;
	while (max_key > 0) {
		max_key >>= 8;
		passes++;
	}
	if (passes == 0) {
		passes = 1;
	}
	int64_t *ik = keys, *ok = aux_k;
	double *iv = vals, *ov = aux_v;
	for (int p = 0; p < passes; p++) {
		int64_t count[256];
		memset(count, 0, sizeof(count));
		int shift = 8 * p;
		for (int64_t i = 0; i < n; i++) {
			count[((uint64_t) ik[i] >> shift) & 0xff]++;
		}
		for (int d = 1; d < 256; d++) {
			count[d] += count[d - 1];
		}
		/* stable distribution from the back: src/mm/mm_utils.c:1347-1364 */
		for (int64_t i = n - 1; i >= 0; i--) {
			int64_t pos = --count[((uint64_t) ik[i] >> shift) & 0xff];
			ok[pos] = ik[i];
			ov[pos] = iv[i];
		}
		int64_t *tk = ik; ik = ok; ok = tk;
		double *tv = iv; iv = ov; ov = tv;
	}
	if (ik != keys) {
		memcpy(keys, ik, sizeof(int64_t) * n);
		memcpy(vals, iv, sizeof(double) * n);
	}
}

/* Hash numeric for one row: probe and accumulate, then emit occupied slots
 * in slot order (ams_hash_numc_krnl src/ams/ams_utils.c:238-309,
 * hybacc_hash_krnl :956-1019). */
static void orc_hash_numc_row(const orc_csr *A, const orc_csr *B, int64_t i, int64_t flp,
	int64_t *check, double *value, int64_t *out_cols, double *out_vals) {
	int64_t size = orc_table_size(flp, B->num_col);
	memset(check, -1, sizeof(int64_t) * size);
	for (int64_t ja = A->row_ptrs[i]; ja < A->row_ptrs[i + 1]; ja++) {
		int64_t k = A->cols[ja];
		double av = A->rats[ja];
		for (int64_t jb = B->row_ptrs[k]; jb < B->row_ptrs[k + 1]; jb++) {
			int64_t key = B->cols[jb];
			double t = av * B->rats[jb];
			int64_t h = orc_hash(key, size);
			for (;;) {
				if (check[h] == key) {
					value[h] += t;
					break;
				} else if (check[h] == -1) {
					check[h] = key;
					value[h] = t;
					break;
				}
				h = (h + 1) & (size - 1);
			}
		}
	}
	int64_t w = 0;
	for (int64_t s = 0; s < size; s++) {
		if (check[s] != -1) {
			out_cols[w] = check[s];
			out_vals[w] = value[s];
			w++;
		}
	}
}

/* ESC numeric for one row: expand, radix sort, compress adjacent equal keys
 * (ams_hsersc_numc_krnl src/ams/ams_utils.c:399-456, hybacc_hsersc_krnl
 * :1023-1075).  The reference compresses with val = old*flag + new
 * (:452-455); this restatement starts a fresh sum on a new key, which is the
 * same for finite values. */
static void orc_esc_numc_row(const orc_csr *A, const orc_csr *B, int64_t i,
	int64_t *ek, double *ev, int64_t *ak, double *av_, int64_t *out_cols, double *out_vals) {
	int64_t n = 0;
	for (int64_t ja = A->row_ptrs[i]; ja < A->row_ptrs[i + 1]; ja++) {
		int64_t k = A->cols[ja];
		double av = A->rats[ja];
		for (int64_t jb = B->row_ptrs[k]; jb < B->row_ptrs[k + 1]; jb++) {
			ek[n] = B->cols[jb];
			ev[n] = av * B->rats[jb];
			n++;
		}
	}
	if (n == 0) {
		return;
	}
	orc_radix_sort_kv(ek, ev, ak, av_, n);
	int64_t w = 0;
	out_cols[0] = ek[0];
	out_vals[0] = ev[0];
	for (int64_t l = 1; l < n; l++) {
		if (ek[l] == ek[l - 1]) {
			out_vals[w] += ev[l];
		} else {
			w++;
			out_cols[w] = ek[l];
			out_vals[w] = ev[l];
		}
	}
}

static int cmp_kv_col(const void *a, const void *b) {
	const int64_t ka = *(const int64_t *) a, kb = *(const int64_t *) b;
	return (ka > kb) - (ka < kb);
}

void orc_sort_rows(orc_csr *C) {
	#pragma omp parallel
	{
		int64_t cap = 0;
		int64_t *tmp = NULL;
		#pragma omp for schedule(dynamic, 256)
		for (int64_t i = 0; i < C->num_row; i++) {
			int64_t s = C->row_ptrs[i], e = C->row_ptrs[i + 1], n = e - s;
			if (n < 2) {
				continue;
			}
			if (n > cap) {
				free(tmp);
				cap = n;
				tmp = (int64_t *) malloc(sizeof(int64_t) * 2 * cap);
			}
			for (int64_t j = 0; j < n; j++) {
				double v = C->rats[s + j];
				tmp[2 * j] = C->cols[s + j];
				memcpy(&tmp[2 * j + 1], &v, sizeof(double));
			}
			qsort(tmp, n, 2 * sizeof(int64_t), cmp_kv_col);
			for (int64_t j = 0; j < n; j++) {
				C->cols[s + j] = tmp[2 * j];
				memcpy(&C->rats[s + j], &tmp[2 * j + 1], sizeof(double));
			}
		}
		free(tmp);
	}
}

int64_t orc_spgemm(const orc_csr *A, const orc_csr *B, orc_csr *C, int algo,
	double acc_thres, int sort_rows) {
	int64_t m = A->num_row;
	memset(C, 0, sizeof(orc_csr));
	C->num_row = m;
	C->num_col = B->num_col;
	int64_t *row_flp = (int64_t *) calloc(m > 0 ? m : 1, sizeof(int64_t));
	int64_t *row_nz = (int64_t *) calloc(m > 0 ? m : 1, sizeof(int64_t));
	C->row_ptrs = (int64_t *) calloc(m + 1, sizeof(int64_t));
	orc_flp_populate(A, B, row_flp);
	int64_t total_flp = 0, max_flp = 0;
	for (int64_t i = 0; i < m; i++) {
		total_flp += row_flp[i];
		if (row_flp[i] > max_flp) {
			max_flp = row_flp[i];
		}
	}
	orc_hash_symb(A, B, row_flp, row_nz);
	orc_scan(C->row_ptrs, row_nz, m + 1);
	C->num_nnz = C->row_ptrs[m];
	C->cols = (int64_t *) malloc(sizeof(int64_t) * (C->num_nnz > 0 ? C->num_nnz : 1));
	C->rats = (double *) malloc(sizeof(double) * (C->num_nnz > 0 ? C->num_nnz : 1));
	int64_t cap = orc_next_pow2(B->num_col > 0 ? B->num_col : 1);
	int64_t esc_cap = max_flp > 0 ? max_flp : 1;
	#pragma omp parallel
	{
		int64_t *check = NULL, *ek = NULL, *ak = NULL;
		double *value = NULL, *ev = NULL, *av = NULL;
		if (algo != ORC_HSERSC) {
			check = (int64_t *) malloc(sizeof(int64_t) * cap);
			value = (double *) malloc(sizeof(double) * cap);
		}
		if (algo != ORC_HASH) {
			ek = (int64_t *) malloc(sizeof(int64_t) * esc_cap);
			ak = (int64_t *) malloc(sizeof(int64_t) * esc_cap);
			ev = (double *) malloc(sizeof(double) * esc_cap);
			av = (double *) malloc(sizeof(double) * esc_cap);
		}
		#pragma omp for schedule(dynamic, 64)
		for (int64_t i = 0; i < m; i++) {
			if (row_flp[i] <= 0) {
				continue;
			}
			int64_t off = C->row_ptrs[i];
			int use_esc;
			if (algo == ORC_HASH) {
				use_esc = 0;
			} else if (algo == ORC_HSERSC) {
				use_esc = 1;
			} else {
				/* per-row choice: src/ams/ams_utils.c:1139-1149 */
				double cf = (double) row_flp[i] / (double) (C->row_ptrs[i + 1] - C->row_ptrs[i]);
				use_esc = cf < acc_thres;
			}
			if (use_esc) {
				orc_esc_numc_row(A, B, i, ek, ev, ak, av, C->cols + off, C->rats + off);
			} else {
				orc_hash_numc_row(A, B, i, row_flp[i], check, value, C->cols + off, C->rats + off);
			}
		}
		free(check); free(value); free(ek); free(ak); free(ev); free(av);
	}
	if (sort_rows) {
		orc_sort_rows(C);
	}
	free(row_flp);
	free(row_nz);
	return total_flp;
}

/* lower_bound over int64 (src/mm/mm_utils.c:963-975). */
static int64_t orc_lower_bound(const int64_t *a, int64_t n, int64_t v) {
	int64_t lo = 0, hi = n;
	while (lo < hi) {
		int64_t mid = lo + (hi - lo) / 2;
		if (a[mid] < v) {
			lo = mid + 1;
		} else {
			hi = mid;
		}
	}
	return lo;
}

typedef struct {
	double cf;
	int64_t idx;
} orc_morsel_key;

static int cmp_morsel(const void *a, const void *b) {
	const orc_morsel_key *x = (const orc_morsel_key *) a, *y = (const orc_morsel_key *) b;
	int c = (x->cf > y->cf) - (x->cf < y->cf);
	if (c) {
		return c;
	}
	return (x->idx > y->idx) - (x->idx < y->idx);
}

int64_t orc_pack_morsels(int64_t num_row, const int64_t *ps_weight, const int64_t *row_flp,
	const int64_t *ps_flp, int64_t morsel, double prt, int64_t *bounds, double *cf,
	int64_t *maxflp, int64_t *order, int64_t *low_head, int64_t *high_tail) {
	int64_t total = ps_weight[num_row] / morsel;
	if (total <= 0) {
		*low_head = 0;
		*high_tail = 0;
		return 0;
	}
	bounds[0] = 0;
	for (int64_t j = 0; j < total; j++) {
		bounds[j + 1] = orc_lower_bound(ps_weight, num_row + 1, morsel * (j + 1));
	}
	bounds[total] = num_row;
	int64_t invalid = 0;
	orc_morsel_key *keys = (orc_morsel_key *) malloc(sizeof(orc_morsel_key) * total);
	for (int64_t j = 0; j < total; j++) {
		int64_t s = bounds[j], e = bounds[j + 1];
		if (e > s) {
			cf[j] = (double) (ps_flp[e] - ps_flp[s]) / (double) (ps_weight[e] - ps_weight[s]);
			int64_t mx = row_flp[s];
			for (int64_t r = s + 1; r < e; r++) {
				mx = row_flp[r] > mx ? row_flp[r] : mx;
			}
			maxflp[j] = mx;
		} else {
			cf[j] = 0.0;
			maxflp[j] = 0;
			invalid++;
		}
		keys[j].cf = cf[j];
		keys[j].idx = j;
	}
	qsort(keys, total, sizeof(orc_morsel_key), cmp_morsel);
	for (int64_t j = 0; j < total; j++) {
		order[j] = keys[j].idx;
	}
	free(keys);
	*low_head = invalid;
	*high_tail = (int64_t) ((double) (total - invalid) * prt + (double) invalid);
	return total;
}

void orc_free(orc_csr *C) {
	free(C->row_ptrs);
	free(C->cols);
	free(C->rats);
	memset(C, 0, sizeof(orc_csr));
}

/* SplitMix64 finaliser (Steele, Lea, Flood 2014), as the casgemm digests use it. */
static uint64_t orc_mix64(uint64_t z) {
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

uint64_t orc_row_digests(const orc_csr *C, int64_t row_offset, uint64_t *row_digests) {
	uint64_t total = 0;
	#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : total)
	for (int64_t i = 0; i < C->num_row; i++) {
		int64_t s = C->row_ptrs[i], e = C->row_ptrs[i + 1];
		uint64_t h = 0;
		for (int64_t j = s; j < e; j++) {
			uint64_t bits;
			memcpy(&bits, &C->rats[j], sizeof(bits));
			h += orc_mix64((uint64_t) C->cols[j] * 0x9E3779B97F4A7C15ull + (uint64_t) (j - s)) ^
				orc_mix64(bits + 0x632BE59BD9B4E019ull);
		}
		if (row_digests) {
			row_digests[i] = h;
		}
		total += orc_mix64(h + (uint64_t) (i + row_offset));
	}
	return total;
}
