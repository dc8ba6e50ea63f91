/*
 * casgemm data layer (declarations and contracts in include/casgemm_data.h).
 *
 * Seeded generators written from the R-MAT definition (Chakrabarti, Zhan,
 * Faloutsos, SDM 2004) and from the Zipf laws the benchmark configurations
 * state; the reference's PaRMAT is unseeded (std::random_device,
 * PaRMAT/src/GraphGen_sorted.cpp:27-28) and is not used.  Random numbers are
 * counter-based (SplitMix64 of a per-item counter), so every output is a pure
 * function of the parameters and the seed, whatever the thread count.
 */
#include "casgemm_data.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* SplitMix64 finaliser (Steele, Lea, Flood, OOPSLA 2014). */
static inline uint64_t cas_mix64(uint64_t z) {
	z += 0x9E3779B97F4A7C15ULL;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
	return z ^ (z >> 31);
}

/* Stream of 64-bit draws for item `idx` of generator `stream`. */
typedef struct {
	uint64_t s;
} cas_rng;

static inline cas_rng cas_rng_at(uint64_t seed, uint64_t stream, uint64_t idx) {
	cas_rng r;
	r.s = cas_mix64(cas_mix64(seed ^ (stream * 0xD1342543DE82EF95ULL)) + idx * 0x9E3779B97F4A7C15ULL);
	return r;
}

static inline uint64_t cas_rng_next(cas_rng *r) {
	r->s += 0x9E3779B97F4A7C15ULL;
	uint64_t z = r->s;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
	return z ^ (z >> 31);
}

/* uniform double in [0, 1) with 53 random bits */
static inline double cas_rng_unit(cas_rng *r) {
	return (double) (cas_rng_next(r) >> 11) * (1.0 / 9007199254740992.0);
}

static int cmp_i32(const void *a, const void *b) {
	int32_t x = *(const int32_t *) a, y = *(const int32_t *) b;
	return (x > y) - (x < y);
}

static void sort_i32(int32_t *a, int64_t n) {
	if (n < 2) {
		return;
	}
	if (n <= 32) {
		for (int64_t i = 1; i < n; i++) {
			int32_t v = a[i];
			int64_t j = i - 1;
			while (j >= 0 && a[j] > v) {
				a[j + 1] = a[j];
				j--;
			}
			a[j + 1] = v;
		}
		return;
	}
	qsort(a, (size_t) n, sizeof(int32_t), cmp_i32);
}

/* ------------------------------------------------------------------ R-MAT */

#define RMAT_INVALID UINT64_MAX
#define RMAT_BUCKET_BITS 12
#define RMAT_NBUCKET (1 << RMAT_BUCKET_BITS)

/* One candidate edge: the quadrant is drawn at each of `scale` levels, from
 * the most significant bit down, with 32-bit thresholds for a, a+b, a+b+c. */
static inline uint64_t rmat_candidate(uint64_t seed, uint64_t e, int scale,
	uint32_t t1, uint32_t t2, uint32_t t3) {
	cas_rng r = cas_rng_at(seed, 1, e);
	uint64_t u = 0, v = 0;
	uint64_t bits = 0;
	int have = 0;
	for (int l = 0; l < scale; l++) {
		if (have == 0) {
			bits = cas_rng_next(&r);
			have = 2;
		}
		uint32_t x = (uint32_t) bits;
		bits >>= 32;
		have--;
		int q = x < t1 ? 0 : (x < t2 ? 1 : (x < t3 ? 2 : 3));
		u = (u << 1) | (uint64_t) (q >> 1);
		v = (v << 1) | (uint64_t) (q & 1);
	}
	if (u == v) {
		return RMAT_INVALID;
	}
	uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
	return (lo << 32) | hi;
}

static inline uint32_t rmat_bucket(uint64_t key) {
	return (uint32_t) (cas_mix64(key) >> (64 - RMAT_BUCKET_BITS));
}

int cas_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
	int64_t *row_ptrs, int32_t *cols) {
	if (scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) {
		return -1;
	}
	const int64_t n = (int64_t) 1 << scale;
	const int64_t n_edges = (int64_t) edge_factor * n;
	if (n_edges > n * (n - 1) / 2) {
		return -1;
	}
	const double two32 = 4294967296.0;
	uint32_t t1 = (uint32_t) fmin(a * two32, 4294967295.0);
	uint32_t t2 = (uint32_t) fmin((a + b) * two32, 4294967295.0);
	uint32_t t3 = (uint32_t) fmin((a + b + c) * two32, 4294967295.0);
	int nthreads = omp_get_max_threads();

	int64_t n_cand = n_edges + n_edges / 16 + 1024;
	uint64_t *acc_keys = NULL;
	int64_t n_acc = 0;
	for (int attempt = 0; attempt < 64; attempt++) {
		uint64_t *keys = (uint64_t *) malloc(sizeof(uint64_t) * n_cand);
		int64_t *bcount = (int64_t *) calloc((size_t) nthreads * RMAT_NBUCKET, sizeof(int64_t));
		int64_t *bstart = (int64_t *) malloc(sizeof(int64_t) * (RMAT_NBUCKET + 1));
		uint64_t *bkey = (uint64_t *) malloc(sizeof(uint64_t) * n_cand);
		int64_t *bidx = (int64_t *) malloc(sizeof(int64_t) * n_cand);
		uint8_t *first = (uint8_t *) calloc((size_t) (n_cand + 7) / 8, 1);
		int64_t *ndist = (int64_t *) calloc(RMAT_NBUCKET, sizeof(int64_t));
		if (!keys || !bcount || !bstart || !bkey || !bidx || !first || !ndist) {
			free(keys); free(bcount); free(bstart); free(bkey); free(bidx); free(first); free(ndist);
			return -1;
		}
		/* candidates, and per-thread bucket counts over contiguous ranges */
		#pragma omp parallel num_threads(nthreads)
		{
			int t = omp_get_thread_num();
			int64_t lo = n_cand * t / nthreads, hi = n_cand * (t + 1) / nthreads;
			int64_t *cnt = bcount + (size_t) t * RMAT_NBUCKET;
			for (int64_t e = lo; e < hi; e++) {
				uint64_t k = rmat_candidate(seed, (uint64_t) e, scale, t1, t2, t3);
				keys[e] = k;
				if (k != RMAT_INVALID) {
					cnt[rmat_bucket(k)]++;
				}
			}
		}
		/* bucket-major, thread-minor offsets: inside a bucket, candidates stay
		 * in increasing candidate order */
		int64_t run = 0;
		for (int bk = 0; bk < RMAT_NBUCKET; bk++) {
			bstart[bk] = run;
			for (int t = 0; t < nthreads; t++) {
				int64_t cnum = bcount[(size_t) t * RMAT_NBUCKET + bk];
				bcount[(size_t) t * RMAT_NBUCKET + bk] = run;
				run += cnum;
			}
		}
		bstart[RMAT_NBUCKET] = run;
		#pragma omp parallel num_threads(nthreads)
		{
			int t = omp_get_thread_num();
			int64_t lo = n_cand * t / nthreads, hi = n_cand * (t + 1) / nthreads;
			int64_t *pos = bcount + (size_t) t * RMAT_NBUCKET;
			for (int64_t e = lo; e < hi; e++) {
				uint64_t k = keys[e];
				if (k != RMAT_INVALID) {
					int64_t p = pos[rmat_bucket(k)]++;
					bkey[p] = k;
					bidx[p] = e;
				}
			}
		}
		free(keys);
		/* first occurrence of every distinct key, per bucket */
		#pragma omp parallel for schedule(dynamic, 8) num_threads(nthreads)
		for (int bk = 0; bk < RMAT_NBUCKET; bk++) {
			int64_t s = bstart[bk], e = bstart[bk + 1], len = e - s;
			if (len == 0) {
				continue;
			}
			int64_t cap = 16;
			while (cap < 2 * len) {
				cap <<= 1;
			}
			uint64_t *set = (uint64_t *) malloc(sizeof(uint64_t) * cap);
			memset(set, 0xff, sizeof(uint64_t) * cap);
			int64_t w = s;
			for (int64_t p = s; p < e; p++) {
				uint64_t k = bkey[p];
				uint64_t h = cas_mix64(k ^ 0x5bd1e995ULL) & (uint64_t) (cap - 1);
				for (;;) {
					if (set[h] == k) {
						break;
					}
					if (set[h] == RMAT_INVALID) {
						set[h] = k;
						bkey[w] = k;
						bidx[w] = bidx[p];
						w++;
						int64_t fi = bidx[p];
						__atomic_fetch_or(&first[fi >> 3], (uint8_t) (1u << (fi & 7)), __ATOMIC_RELAXED);
						break;
					}
					h = (h + 1) & (uint64_t) (cap - 1);
				}
			}
			ndist[bk] = w - s;
			free(set);
		}
		int64_t total = 0;
		for (int bk = 0; bk < RMAT_NBUCKET; bk++) {
			total += ndist[bk];
		}
		if (total < n_edges) {
			free(bcount); free(bstart); free(bkey); free(bidx); free(first); free(ndist);
			n_cand += (n_edges - total) * 2 + n_edges / 8 + 1024;
			continue;
		}
		/* cut-off: candidate index at which the n_edges-th distinct edge first
		 * appears (sequential acceptance in candidate order) */
		int64_t seen = 0, cut = -1;
		for (int64_t byte = 0; byte < (n_cand + 7) / 8 && cut < 0; byte++) {
			int pc = __builtin_popcount(first[byte]);
			if (seen + pc < n_edges) {
				seen += pc;
				continue;
			}
			for (int bit = 0; bit < 8; bit++) {
				if ((first[byte] >> bit) & 1) {
					seen++;
					if (seen == n_edges) {
						cut = byte * 8 + bit;
						break;
					}
				}
			}
		}
		acc_keys = (uint64_t *) malloc(sizeof(uint64_t) * n_edges);
		n_acc = 0;
		for (int bk = 0; bk < RMAT_NBUCKET; bk++) {
			int64_t s = bstart[bk];
			for (int64_t p = s; p < s + ndist[bk]; p++) {
				if (bidx[p] <= cut) {
					acc_keys[n_acc++] = bkey[p];
				}
			}
		}
		free(bcount); free(bstart); free(bkey); free(bidx); free(first); free(ndist);
		break;
	}
	if (!acc_keys || n_acc != n_edges) {
		free(acc_keys);
		return -1;
	}
	/* symmetrise into CSR */
	int64_t *deg = (int64_t *) calloc((size_t) n, sizeof(int64_t));
	#pragma omp parallel for num_threads(nthreads)
	for (int64_t e = 0; e < n_edges; e++) {
		uint64_t k = acc_keys[e];
		__atomic_fetch_add(&deg[k >> 32], 1, __ATOMIC_RELAXED);
		__atomic_fetch_add(&deg[k & 0xffffffffULL], 1, __ATOMIC_RELAXED);
	}
	row_ptrs[0] = 0;
	for (int64_t i = 0; i < n; i++) {
		row_ptrs[i + 1] = row_ptrs[i] + deg[i];
		deg[i] = row_ptrs[i];
	}
	#pragma omp parallel for num_threads(nthreads)
	for (int64_t e = 0; e < n_edges; e++) {
		uint64_t k = acc_keys[e];
		int64_t lo = (int64_t) (k >> 32), hi = (int64_t) (k & 0xffffffffULL);
		cols[__atomic_fetch_add(&deg[lo], 1, __ATOMIC_RELAXED)] = (int32_t) hi;
		cols[__atomic_fetch_add(&deg[hi], 1, __ATOMIC_RELAXED)] = (int32_t) lo;
	}
	#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads)
	for (int64_t i = 0; i < n; i++) {
		sort_i32(cols + row_ptrs[i], row_ptrs[i + 1] - row_ptrs[i]);
	}
	free(deg);
	free(acc_keys);
	return 0;
}

/* ------------------------------------------------------------------- Zipf */

static int64_t zipf_deg_sum(int64_t num_row, int64_t amax, double row_s, double q, int64_t *deg) {
	int64_t s = 0;
	for (int64_t r = 1; r <= num_row; r++) {
		double d = (double) amax * pow((1.0 + q) / ((double) r + q), row_s);
		int64_t di = (int64_t) llround(d);
		if (di < 1) {
			di = 1;
		}
		if (deg) {
			deg[r - 1] = di;
		}
		s += di;
	}
	return s;
}

double cas_zipf_row_degrees(int64_t num_row, int64_t amax, double row_s, int64_t target_nnz,
	int64_t *deg) {
	if (num_row < 1 || amax < 1 || target_nnz < num_row) {
		return -1.0;
	}
	double lo = 0.0, hi = 1.0;
	while (zipf_deg_sum(num_row, amax, row_s, hi, NULL) < target_nnz && hi < 1e12) {
		hi *= 2.0;
	}
	for (int it = 0; it < 200; it++) {
		double mid = 0.5 * (lo + hi);
		if (zipf_deg_sum(num_row, amax, row_s, mid, NULL) < target_nnz) {
			lo = mid;
		} else {
			hi = mid;
		}
	}
	double q = hi;
	zipf_deg_sum(num_row, amax, row_s, q, deg);
	return q;
}

int64_t cas_gen_zipf(int64_t num_row, int64_t num_col, int64_t amax, double row_s,
	int64_t target_nnz, double col_s, double col_q, uint64_t seed,
	int64_t *row_ptrs, int32_t *cols) {
	if (num_col < 1 || num_col > INT32_MAX || amax > num_col) {
		return -1;
	}
	int64_t *deg = (int64_t *) malloc(sizeof(int64_t) * num_row);
	if (cas_zipf_row_degrees(num_row, amax, row_s, target_nnz, deg) < 0) {
		free(deg);
		return -1;
	}
	/* seeded Fisher-Yates shuffle of the row order */
	cas_rng pr = cas_rng_at(seed, 2, 0);
	for (int64_t i = num_row - 1; i > 0; i--) {
		int64_t j = (int64_t) (cas_rng_next(&pr) % (uint64_t) (i + 1));
		int64_t t = deg[i];
		deg[i] = deg[j];
		deg[j] = t;
	}
	row_ptrs[0] = 0;
	for (int64_t i = 0; i < num_row; i++) {
		row_ptrs[i + 1] = row_ptrs[i] + deg[i];
	}
	int64_t nnz = row_ptrs[num_row];
	if (cols == NULL) {
		free(deg);
		return nnz;
	}
	/* column CDF of p_k proportional to (k + col_q)^-col_s, k = 1..num_col */
	double *cdf = (double *) malloc(sizeof(double) * num_col);
	double acc = 0.0;
	for (int64_t k = 0; k < num_col; k++) {
		acc += pow((double) (k + 1) + col_q, -col_s);
		cdf[k] = acc;
	}
	for (int64_t k = 0; k < num_col; k++) {
		cdf[k] /= acc;
	}
	cdf[num_col - 1] = 1.0;
	int failed = 0;
	#pragma omp parallel
	{
		int64_t cap = 0;
		int32_t *set = NULL;
		#pragma omp for schedule(dynamic, 64)
		for (int64_t i = 0; i < num_row; i++) {
			int64_t d = deg[i];
			int64_t need = 16;
			while (need < 2 * d) {
				need <<= 1;
			}
			if (need > cap) {
				free(set);
				cap = need;
				set = (int32_t *) malloc(sizeof(int32_t) * cap);
			}
			memset(set, 0xff, sizeof(int32_t) * need);
			cas_rng r = cas_rng_at(seed, 3, (uint64_t) i);
			int32_t *out = cols + row_ptrs[i];
			int64_t got = 0, draws = 0;
			while (got < d) {
				if (++draws > 64 * d + 1000000) {
					failed = 1;
					break;
				}
				double u = cas_rng_unit(&r);
				int64_t lo = 0, hi = num_col - 1;
				while (lo < hi) {
					int64_t mid = (lo + hi) >> 1;
					if (cdf[mid] > u) {
						hi = mid;
					} else {
						lo = mid + 1;
					}
				}
				int32_t k = (int32_t) lo;
				uint64_t h = cas_mix64((uint64_t) k) & (uint64_t) (need - 1);
				for (;;) {
					if (set[h] == k) {
						break;
					}
					if (set[h] < 0) {
						set[h] = k;
						out[got++] = k;
						break;
					}
					h = (h + 1) & (uint64_t) (need - 1);
				}
			}
			sort_i32(out, d);
		}
		free(set);
	}
	free(cdf);
	free(deg);
	return failed ? -1 : nnz;
}

void cas_gen_int_values(int64_t nnz, int32_t lo, int32_t hi, uint64_t seed, int32_t *vals) {
	uint64_t span = (uint64_t) ((int64_t) hi - (int64_t) lo + 1);
	#pragma omp parallel for
	for (int64_t e = 0; e < nnz; e++) {
		cas_rng r = cas_rng_at(seed, 4, (uint64_t) e);
		vals[e] = (int32_t) ((int64_t) lo + (int64_t) (cas_rng_next(&r) % span));
	}
}

/* -------------------------------------------------------- CSR utilities */

int cas_csr_transpose_host(int64_t num_row, int64_t num_col, const int64_t *row_ptrs,
	const int32_t *cols, const void *vals, int val_bytes,
	int64_t *t_row_ptrs, int32_t *t_cols, void *t_vals) {
	if (vals && val_bytes != 4 && val_bytes != 8) {
		return -1;
	}
	int64_t nnz = row_ptrs[num_row];
	memset(t_row_ptrs, 0, sizeof(int64_t) * (num_col + 1));
	for (int64_t e = 0; e < nnz; e++) {
		t_row_ptrs[cols[e] + 1]++;
	}
	for (int64_t j = 0; j < num_col; j++) {
		t_row_ptrs[j + 1] += t_row_ptrs[j];
	}
	int64_t *cur = (int64_t *) malloc(sizeof(int64_t) * (num_col > 0 ? num_col : 1));
	memcpy(cur, t_row_ptrs, sizeof(int64_t) * num_col);
	for (int64_t i = 0; i < num_row; i++) {
		for (int64_t e = row_ptrs[i]; e < row_ptrs[i + 1]; e++) {
			int64_t p = cur[cols[e]]++;
			t_cols[p] = (int32_t) i;
			if (vals) {
				memcpy((char *) t_vals + p * val_bytes, (const char *) vals + e * val_bytes, (size_t) val_bytes);
			}
		}
	}
	free(cur);
	return 0;
}

int64_t cas_intprod_host(int64_t num_row, const int64_t *a_row_ptrs, const int32_t *a_cols,
	const int64_t *b_row_ptrs) {
	int64_t total = 0;
	#pragma omp parallel for reduction(+:total) schedule(static, 4096)
	for (int64_t i = 0; i < num_row; i++) {
		for (int64_t e = a_row_ptrs[i]; e < a_row_ptrs[i + 1]; e++) {
			int32_t k = a_cols[e];
			total += b_row_ptrs[k + 1] - b_row_ptrs[k];
		}
	}
	return total;
}

/* ------------------------------------------------------------ MatrixMarket */

static const char *skip_ws(const char *p, const char *end) {
	while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) {
		p++;
	}
	return p;
}

static const char *parse_i64(const char *p, const char *end, int64_t *out, int *ok) {
	p = skip_ws(p, end);
	int neg = 0;
	if (p < end && (*p == '-' || *p == '+')) {
		neg = *p == '-';
		p++;
	}
	if (p >= end || *p < '0' || *p > '9') {
		*ok = 0;
		return p;
	}
	int64_t v = 0;
	while (p < end && *p >= '0' && *p <= '9') {
		v = v * 10 + (*p - '0');
		p++;
	}
	*out = neg ? -v : v;
	*ok = 1;
	return p;
}

int64_t cas_mtx_read(const char *path, int64_t *num_row, int64_t *num_col,
	int64_t *row_ptrs, int32_t *cols, double *vals) {
	FILE *f = fopen(path, "rb");
	if (!f) {
		return -1;
	}
	fseek(f, 0, SEEK_END);
	long sz = ftell(f);
	fseek(f, 0, SEEK_SET);
	char *buf = (char *) malloc((size_t) sz + 1);
	if (!buf || fread(buf, 1, (size_t) sz, f) != (size_t) sz) {
		free(buf);
		fclose(f);
		return -1;
	}
	fclose(f);
	buf[sz] = '\0';
	const char *p = buf, *end = buf + sz;
	int symmetric = 0, header = 0;
	int64_t hdr_nnz = 0, cnt = 0;
	int64_t *ri = NULL, *ci = NULL;
	int64_t cap = 0;
	while (p < end) {
		const char *nl = memchr(p, '\n', (size_t) (end - p));
		const char *le = nl ? nl : end;
		if (le > p && p[0] == '%') {
			/* mtx2trpl: a comment containing "symmetric" marks the file
			 * symmetric (src/mm/mm_utils.c:509-514) */
			for (const char *s = p; s + 9 <= le; s++) {
				if (memcmp(s, "symmetric", 9) == 0) {
					symmetric = 1;
					break;
				}
			}
		} else if (skip_ws(p, le) < le) {
			int ok1, ok2, ok3;
			int64_t r, c, z;
			const char *q = parse_i64(p, le, &r, &ok1);
			q = parse_i64(q, le, &c, &ok2);
			if (!header) {
				q = parse_i64(q, le, &z, &ok3);
				if (!ok1 || !ok2 || !ok3) {
					free(buf);
					return -1;
				}
				*num_row = r;
				*num_col = c;
				hdr_nnz = z;
				header = 1;
				cap = symmetric ? 2 * hdr_nnz : hdr_nnz;
				ri = (int64_t *) malloc(sizeof(int64_t) * (cap > 0 ? cap : 1));
				ci = (int64_t *) malloc(sizeof(int64_t) * (cap > 0 ? cap : 1));
			} else {
				if (!ok1 || !ok2) {
					free(buf); free(ri); free(ci);
					return -1;
				}
				/* value: absent -> 1.0; explicit zero -> dropped
				 * (src/mm/mm_utils.c:543-559); otherwise forced to 1.0 (:561) */
				q = skip_ws(q, le);
				int zero = 0;
				if (q < le) {
					char tmp[64];
					size_t L = (size_t) (le - q) < 63 ? (size_t) (le - q) : 63;
					memcpy(tmp, q, L);
					tmp[L] = '\0';
					zero = strtod(tmp, NULL) == 0.0;
				}
				if (!zero) {
					if (cnt + 2 > cap) {
						cap = cap * 2 + 16;
						ri = (int64_t *) realloc(ri, sizeof(int64_t) * cap);
						ci = (int64_t *) realloc(ci, sizeof(int64_t) * cap);
					}
					ri[cnt] = r - 1;
					ci[cnt] = c - 1;
					cnt++;
					if (symmetric && r != c) {
						ri[cnt] = c - 1;
						ci[cnt] = r - 1;
						cnt++;
					}
				}
			}
		}
		p = nl ? nl + 1 : end;
	}
	free(buf);
	if (!header) {
		return -1;
	}
	if (cols == NULL) {
		free(ri);
		free(ci);
		return cnt;
	}
	/* sort by (row, col), duplicates kept (src/mm/mm_utils.c:600-604, 650-692) */
	memset(row_ptrs, 0, sizeof(int64_t) * (*num_row + 1));
	for (int64_t e = 0; e < cnt; e++) {
		row_ptrs[ri[e] + 1]++;
	}
	for (int64_t i = 0; i < *num_row; i++) {
		row_ptrs[i + 1] += row_ptrs[i];
	}
	int64_t *cur = (int64_t *) malloc(sizeof(int64_t) * (*num_row > 0 ? *num_row : 1));
	memcpy(cur, row_ptrs, sizeof(int64_t) * (*num_row));
	for (int64_t e = 0; e < cnt; e++) {
		cols[cur[ri[e]]++] = (int32_t) ci[e];
	}
	free(cur);
	#pragma omp parallel for schedule(dynamic, 1024)
	for (int64_t i = 0; i < *num_row; i++) {
		sort_i32(cols + row_ptrs[i], row_ptrs[i + 1] - row_ptrs[i]);
	}
	if (vals) {
		for (int64_t e = 0; e < cnt; e++) {
			vals[e] = 1.0;
		}
	}
	free(ri);
	free(ci);
	return cnt;
}

static char *put_u64(char *o, uint64_t v) {
	char t[24];
	int n = 0;
	do {
		t[n++] = (char) ('0' + v % 10);
		v /= 10;
	} while (v);
	while (n) {
		*o++ = t[--n];
	}
	return o;
}

int cas_mtx_write(const char *path, int64_t num_row, int64_t num_col, const int64_t *row_ptrs,
	const int32_t *cols, int symmetric) {
	FILE *f = fopen(path, "wb");
	if (!f) {
		return -1;
	}
	int64_t cnt = 0;
	for (int64_t i = 0; i < num_row; i++) {
		for (int64_t e = row_ptrs[i]; e < row_ptrs[i + 1]; e++) {
			if (!symmetric || i <= cols[e]) {
				cnt++;
			}
		}
	}
	/* the reference's header line has one '%' (its format string is "%%...") */
	fputs(symmetric ? "%MatrixMarket matrix coordinate real symmetric\n"
		: "%MatrixMarket matrix coordinate real general\n", f);
	fprintf(f, "%ld %ld %ld\n", (long) num_row, (long) num_col, (long) cnt);
	size_t bcap = 1 << 22;
	char *b = (char *) malloc(bcap + 128);
	char *o = b;
	for (int64_t i = 0; i < num_row; i++) {
		for (int64_t e = row_ptrs[i]; e < row_ptrs[i + 1]; e++) {
			if (symmetric && i > cols[e]) {
				continue;
			}
			o = put_u64(o, (uint64_t) i + 1);
			*o++ = ' ';
			o = put_u64(o, (uint64_t) cols[e] + 1);
			memcpy(o, " 1.000000\n", 10);
			o += 10;
			if ((size_t) (o - b) > bcap) {
				fwrite(b, 1, (size_t) (o - b), f);
				o = b;
			}
		}
	}
	fwrite(b, 1, (size_t) (o - b), f);
	free(b);
	return fclose(f) == 0 ? 0 : -1;
}

/* ------------------------------------------------------- binary CSR cache */

static const char cas_csr_magic[8] = {'C', 'A', 'S', 'C', 'S', 'R', '1', '\0'};

int cas_csr_write_bin(const char *path, int64_t num_row, int64_t num_col, const int64_t *row_ptrs,
	const int32_t *cols, const double *vals) {
	if (!path || num_row < 0 || num_col < 0 || !row_ptrs) {
		return -1;
	}
	const int64_t nnz = row_ptrs[num_row] - row_ptrs[0];
	if (row_ptrs[0] != 0 || nnz < 0 || (nnz > 0 && (!cols || !vals))) {
		return -1;
	}
	FILE *f = fopen(path, "wb");
	if (!f) {
		return -1;
	}
	const int64_t head[3] = {num_row, num_col, nnz};
	int ok = fwrite(cas_csr_magic, 1, 8, f) == 8 && fwrite(head, sizeof(int64_t), 3, f) == 3 &&
		fwrite(row_ptrs, sizeof(int64_t), (size_t) (num_row + 1), f) == (size_t) (num_row + 1) &&
		(nnz == 0 || (fwrite(cols, sizeof(int32_t), (size_t) nnz, f) == (size_t) nnz &&
			fwrite(vals, sizeof(double), (size_t) nnz, f) == (size_t) nnz));
	ok = (fclose(f) == 0) && ok;
	return ok ? 0 : -1;
}

int64_t cas_csr_read_bin(const char *path, int64_t *num_row, int64_t *num_col, int64_t *row_ptrs,
	int32_t *cols, double *vals) {
	if (!path || !num_row || !num_col) {
		return -1;
	}
	FILE *f = fopen(path, "rb");
	if (!f) {
		return -1;
	}
	char magic[8];
	int64_t head[3];
	if (fread(magic, 1, 8, f) != 8 || memcmp(magic, cas_csr_magic, 8) != 0 ||
		fread(head, sizeof(int64_t), 3, f) != 3 || head[0] < 0 || head[1] < 0 || head[2] < 0) {
		fclose(f);
		return -1;
	}
	*num_row = head[0];
	*num_col = head[1];
	const int64_t nnz = head[2];
	if (cols) {
		if (!row_ptrs || (nnz > 0 && !vals) ||
			fread(row_ptrs, sizeof(int64_t), (size_t) (head[0] + 1), f) != (size_t) (head[0] + 1) ||
			(nnz > 0 && (fread(cols, sizeof(int32_t), (size_t) nnz, f) != (size_t) nnz ||
				fread(vals, sizeof(double), (size_t) nnz, f) != (size_t) nnz)) ||
			row_ptrs[0] != 0 || row_ptrs[head[0]] != nnz) {
			fclose(f);
			return -1;
		}
	}
	fclose(f);
	return nnz;
}
