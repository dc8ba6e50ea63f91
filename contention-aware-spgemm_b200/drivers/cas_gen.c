/*
 * Dataset generator for the drivers: writes <dir>/<name>.org.mtx (A) and
 * <dir>/<name>.trs.mtx (B = A^T) from the project's seeded generators, in
 * the MatrixMarket form the reference's rmat_ones writes (trpl2mtx,
 * src/mm/mm_utils.c:610-647).  It replaces the reference's unseeded PaRMAT
 * step (scripts/rmat_preparation.sh:39-48) with a seeded R-MAT.
 *
 *   cas_gen g500 <scale> <edge_factor> [seed]   -> g500_<scale>_<edge_factor>
 *   cas_gen er   <scale> <edge_factor> [seed]   -> er_<scale>_<edge_factor>
 *   cas_gen zipf <name> <rows> <cols> <max_row_nnz> <target_nnz> <col_q> [seed]
 *
 * R-MAT: a=.57 b=.19 c=.19 (g500) or a=b=c=.25 (er), symmetrised, loop- and
 * duplicate-free, written as "symmetric" files (org and trs hold the same
 * matrix).  Zipf bipartite: row degrees Zipf(1.2), columns Zipf(1.4) shifted
 * by col_q, org general and trs its explicit transpose.  Default seed: the
 * scale (R-MAT) or 3 (Zipf).  Output directory: CAS_DATASET_DIR or ./dataset.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "casgemm_data.h"

static int write_pair(const char *dir, const char *name, int64_t nr, int64_t nc, const int64_t *rp,
                      const int32_t *cols, int symmetric) {
	char org[4096], trs[4096];
	snprintf(org, sizeof(org), "%s/%s.org.mtx", dir, name);
	snprintf(trs, sizeof(trs), "%s/%s.trs.mtx", dir, name);
	if (cas_mtx_write(org, nr, nc, rp, cols, symmetric) != 0) return -1;
	if (symmetric) return cas_mtx_write(trs, nr, nc, rp, cols, 1);
	const int64_t nnz = rp[nr];
	int64_t *trp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nc + 1));
	int32_t *tcols = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
	if (!trp || !tcols) return -1;
	int rc = cas_csr_transpose_host(nr, nc, rp, cols, NULL, 8, trp, tcols, NULL);
	if (rc == 0) rc = cas_mtx_write(trs, nc, nr, trp, tcols, 0);
	free(trp);
	free(tcols);
	return rc;
}

static void usage(const char *p) {
	fprintf(stderr,
	        "usage: %s g500|er <scale> <edge_factor> [seed]\n"
	        "       %s zipf <name> <rows> <cols> <max_row_nnz> <target_nnz> <col_q> [seed]\n",
	        p, p);
	exit(1);
}

int main(int argc, char **argv) {
	if (argc < 2) usage(argv[0]);
	const char *dir = getenv("CAS_DATASET_DIR");
	if (!dir || !*dir) dir = "./dataset";
	mkdir(dir, 0755);
	char name[1024];
	if (!strcmp(argv[1], "g500") || !strcmp(argv[1], "er")) {
		if (argc < 4) usage(argv[0]);
		const int scale = atoi(argv[2]), ef = atoi(argv[3]);
		const uint64_t seed = argc > 4 ? strtoull(argv[4], NULL, 10) : (uint64_t)scale;
		const int g500 = !strcmp(argv[1], "g500");
		if (scale < 1 || scale > 30 || ef < 1) usage(argv[0]);
		const int64_t n = (int64_t)1 << scale, nnz = 2 * (int64_t)ef * n;
		int64_t *rp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
		int32_t *cols = (int32_t *)malloc(sizeof(int32_t) * (size_t)nnz);
		if (!rp || !cols) return 1;
		if (cas_gen_rmat(scale, ef, g500 ? 0.57 : 0.25, g500 ? 0.19 : 0.25, g500 ? 0.19 : 0.25, seed, rp, cols) != 0) {
			fprintf(stderr, "R-MAT generation failed\n");
			return 1;
		}
		snprintf(name, sizeof(name), "%s_%d_%d", argv[1], scale, ef);
		if (write_pair(dir, name, n, n, rp, cols, 1) != 0) {
			fprintf(stderr, "writing %s/%s failed\n", dir, name);
			return 1;
		}
		printf("%s/%s: %ld x %ld, nnz %ld\n", dir, name, (long)n, (long)n, (long)nnz);
		free(rp);
		free(cols);
		return 0;
	}
	if (!strcmp(argv[1], "zipf")) {
		if (argc < 8) usage(argv[0]);
		snprintf(name, sizeof(name), "%s", argv[2]);
		const int64_t nr = atoll(argv[3]), nc = atoll(argv[4]), amax = atoll(argv[5]), target = atoll(argv[6]);
		const double col_q = atof(argv[7]);
		const uint64_t seed = argc > 8 ? strtoull(argv[8], NULL, 10) : 3;
		if (nr < 1 || nc < 1 || amax < 1 || amax > nc || target < nr) usage(argv[0]);
		int64_t *rp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nr + 1));
		if (!rp) return 1;
		const int64_t nnz = cas_gen_zipf(nr, nc, amax, 1.2, target, 1.4, col_q, seed, rp, NULL);
		if (nnz < 0) return 1;
		int32_t *cols = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
		if (!cols || cas_gen_zipf(nr, nc, amax, 1.2, target, 1.4, col_q, seed, rp, cols) != nnz) return 1;
		if (write_pair(dir, name, nr, nc, rp, cols, 0) != 0) {
			fprintf(stderr, "writing %s/%s failed\n", dir, name);
			return 1;
		}
		printf("%s/%s: %ld x %ld, nnz %ld\n", dir, name, (long)nr, (long)nc, (long)nnz);
		free(rp);
		free(cols);
		return 0;
	}
	usage(argv[0]);
	return 1;
}
