/*
 * cas_rmat_ones <dataset>: the reference's rmat_ones (src/rmat_ones.c) —
 * an R-MAT edge list <dir>/<dataset>.txt (PaRMAT output: 0-based
 * "u v [w]" lines, each undirected edge once) becomes <dir>/<dataset>.org.mtx
 * and <dir>/<dataset>.trs.mtx with every value 1.0 (txt_transpose,
 * src/mm/mm_utils.c:851-862).  As txt2trpl (src/mm/mm_utils.c:759-840)
 * does: the vertex count is 2^scale from the name <family>_<scale>_<ef>,
 * lines with weight 0 are skipped, each edge is stored in both directions
 * (self-loops are an error), entries are sorted by (row, col), and both
 * files are written "symmetric" (entries with row <= col).  The transpose
 * of a symmetric matrix is itself, so trs holds the same entries.
 * Directory: CAS_DATASET_DIR or ./dataset.  Exit status 1 on failure.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "casgemm_data.h"

static int cmp_u64(const void *a, const void *b) {
	const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
	return x < y ? -1 : x > y;
}

int main(int argc, char **argv) {
	if (argc != 2) {
		fprintf(stderr, "usage: %s <dataset>\n", argv[0]);
		return 1;
	}
	const char *dataset = argv[1];
	const char *dir = getenv("CAS_DATASET_DIR");
	if (!dir || !*dir) dir = "./dataset";
	int scale = 0, ef = 0;
	const char *us = strchr(dataset, '_');
	if (!us || sscanf(us + 1, "%d_%d", &scale, &ef) != 2 || scale < 1 || scale > 30) {
		fprintf(stderr, "dataset name must be <family>_<scale>_<edge_factor>: %s\n", dataset);
		return 1;
	}
	const int64_t n = (int64_t)1 << scale;
	char src[4096], org[4096], trs[4096];
	snprintf(src, sizeof(src), "%s/%s.txt", dir, dataset);
	snprintf(org, sizeof(org), "%s/%s.org.mtx", dir, dataset);
	snprintf(trs, sizeof(trs), "%s/%s.trs.mtx", dir, dataset);
	FILE *f = fopen(src, "r");
	if (!f) {
		fprintf(stderr, "Error opening file, %s\n", src);
		return 1;
	}
	size_t cap = 1 << 20, cnt = 0;
	uint64_t *key = (uint64_t *)malloc(sizeof(uint64_t) * cap);
	char line[4096];
	while (key && fgets(line, sizeof(line), f)) {
		long u, v;
		double w = 1.0;
		const int got = sscanf(line, "%ld %ld %lf", &u, &v, &w);
		if (got == 2) w = 1.0;
		else if (got != 3) {
			fprintf(stderr, "Error reading line: %s\n", line);
			return 1;
		}
		if (w == 0.0) continue;
		if (u < 0 || v < 0 || u >= n || v >= n || u == v) {
			fprintf(stderr, "bad edge %ld %ld for 2^%d vertices\n", u, v, scale);
			return 1;
		}
		if (cnt + 2 > cap) {
			cap *= 2;
			key = (uint64_t *)realloc(key, sizeof(uint64_t) * cap);
			if (!key) break;
		}
		key[cnt++] = ((uint64_t)u << 32) | (uint64_t)v;
		key[cnt++] = ((uint64_t)v << 32) | (uint64_t)u;
	}
	fclose(f);
	if (!key) {
		fprintf(stderr, "host allocation failed\n");
		return 1;
	}
	qsort(key, cnt, sizeof(uint64_t), cmp_u64);
	int64_t *rp = (int64_t *)calloc((size_t)(n + 1), sizeof(int64_t));
	int32_t *cols = (int32_t *)malloc(sizeof(int32_t) * (cnt > 0 ? cnt : 1));
	if (!rp || !cols) return 1;
	for (size_t i = 0; i < cnt; ++i) {
		rp[(key[i] >> 32) + 1]++;
		cols[i] = (int32_t)(key[i] & 0xFFFFFFFFu);
	}
	for (int64_t r = 0; r < n; ++r) rp[r + 1] += rp[r];
	if (cas_mtx_write(org, n, n, rp, cols, 1) != 0 || cas_mtx_write(trs, n, n, rp, cols, 1) != 0) {
		fprintf(stderr, "writing %s failed\n", org);
		return 1;
	}
	printf("%s: %ld x %ld, nnz %ld (edge factor %d)\n", dataset, (long)n, (long)n, (long)cnt, ef);
	free(key);
	free(rp);
	free(cols);
	return 0;
}
