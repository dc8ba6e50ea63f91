/*
 * The three SpGEMM command-line drivers, over the casgemm C ABI.
 *
 * Same process interface as the reference's drivers (src/ams_hashspgemm.c,
 * src/ams_hserscspgemm.c, src/ams_hybaccspgemm.c, main at :222-382 of each):
 *
 *   bin/<driver> <dataset>
 *
 * reads <dir>/<dataset>.org.mtx as A and <dir>/<dataset>.trs.mtx as B (the
 * reference's get_matrix_paths, src/mm/mm_utils.h:63-70, with RMAT_DIR =
 * ./dataset; when the .trs.mtx file is absent, or CAS_TRANSPOSE is 1, B =
 * A^T is made on the device instead, outside the timed phases, as reading
 * the file is), with the reference loader's semantics (raw2csr,
 * src/mm/mm_utils.c:451-692: values forced to 1.0, explicit zeros dropped,
 * symmetric files mirrored, duplicates kept).  It runs the product RUN_NUM
 * times (run 0 is the warm-up), and writes the reference's text to stdout:
 *
 *   CONFIGURATION:\t...                                  (cfg_print, src/mm/mm_utils.c:1540-1605)
 *   <i>th run\tinit_time: ..\tsymb_time: ..\tmgmt_time: ..\tnumc_time: ..\ttotal_time: ..
 *   VERIFYRESULT:\t<nnz>\t<sum of cols>\t<sum of vals>   (IN_VERIFY, runs 1.., with CAS_VERIFY=1)
 *   dataset: ..\tnum_trials: ..\tthread_num: ..\tnuma_mask: ..\tinit_time: .. total_time: ..
 *     \tflop_cnt: ..\tnumc_perf: ..\tperf: ..                (src/ams_hashspgemm.c:366-378)
 *
 * with the same escape colours.  Fields the GPU adds come after the
 * reference's: gflops (2 * flop_cnt / total_time / 1e9), hbm_frac (the
 * Gustavson traffic model 12 nnz(A) + 12 flop + 12 nnz(C) + 16 (m + 1) bytes
 * over total_time, against the HBM peak), device, hbm_peak_gbs.  As in the
 * reference, numc_perf and perf are flop_cnt per second of numc_time /
 * total_time.
 *
 * The CONFIGURATION line carries the reference's fields first, in its order
 * (HASH_CONSTANT .. HYB_THRES), so log parsers keyed on them keep working,
 * then the GPU's (DRIVER, DEVICE, CUDA_DEVICE, SM_COUNT, RUN_NUM).  The
 * reference's fields hold the values of the reference build whose output the
 * driver reproduces, the per-driver settings of scripts/ams_rmat_run.sh:25-36
 * with the build macros of scripts/ams_run_common.sh:20-33, except two that
 * describe this run: THREAD_NUM is the GPU's resident thread count (SMs times
 * threads per SM) and AMS_HIGH_THREAD_NUM the same share of it as the
 * script's 16 or 22 of 64 threads; AMS_ACC_THRES is the value in use.  None
 * of them changes the output: rows are sorted, and the sums are exact.
 *
 * The phases are timed on the device with CUDA events around the work the
 * reference times: A and B are loaded and resident before run 0, C is
 * freed after each run (free_csr).  thread_num reports the GPU's SM count
 * and numa_mask the bit of the CUDA device used.
 *
 * Environment: CAS_DATASET_DIR (default ./dataset), CAS_CSR_CACHE (1: keep
 * and reuse a binary <dataset>.org.csr / .trs.csr beside the .mtx files), CAS_RUN_NUM (default 10,
 * at least 2, the reference's RUN_NUM), CAS_DEVICE (default 0),
 * CAS_VERIFY (1: VERIFYRESULT lines), CAS_ACC_THRES (hybrid threshold,
 * default 2.0 = the R-MAT scripts' value), CAS_PEAK_GBS (HBM bandwidth in
 * GB/s for hbm_frac); without it the driver reads "hbm_gbs" from the JSON
 * file named by CAS_PEAKS_JSON (default ./MEASURED_PEAKS.json, a measured
 * copy bandwidth), and failing that uses 6650, a copy kernel's rate measured
 * on B200 earlier.
 * Failures print a message to stderr and exit with status 1, as the
 * reference's exit(1) does.
 */
#ifndef CAS_DRIVER_H
#define CAS_DRIVER_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "casgemm.h"
#include "casgemm_data.h"

#define CAS_DRIVER_PATH_LEN 4096

static void drv_green(void) { printf("\033[0;32m"); }
static void drv_cyan(void) { printf("\033[0;36m"); }
static void drv_reset(void) { printf("\033[0m"); }

static void drv_die(const char *what) {
	fprintf(stderr, "%s\n", what);
	exit(1);
}

static long drv_env_long(const char *name, long dflt) {
	const char *s = getenv(name);
	return (s && *s) ? strtol(s, NULL, 10) : dflt;
}

static double drv_env_double(const char *name, double dflt) {
	const char *s = getenv(name);
	return (s && *s) ? strtod(s, NULL) : dflt;
}

/* Host CSR from a MatrixMarket file (two-phase cas_mtx_read), or from its
 * binary cache <path without .mtx>.csr when CAS_CSR_CACHE is 1 (written on
 * the first run, read on the later ones). */
static void drv_load(const char *path, cas_csr *M) {
	int64_t nr = 0, nc = 0;
	char bin[CAS_DRIVER_PATH_LEN];
	const int cache = (int)drv_env_long("CAS_CSR_CACHE", 0);
	snprintf(bin, sizeof(bin), "%s", path);
	char *dot = strrchr(bin, '.');
	if (dot && !strcmp(dot, ".mtx")) strcpy(dot, ".csr");
	if (cache) {
		const int64_t bnnz = cas_csr_read_bin(bin, &nr, &nc, NULL, NULL, NULL);
		if (bnnz >= 0) {
			int64_t *rp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nr + 1));
			int32_t *cols = (int32_t *)malloc(sizeof(int32_t) * (size_t)(bnnz > 0 ? bnnz : 1));
			double *vals = (double *)malloc(sizeof(double) * (size_t)(bnnz > 0 ? bnnz : 1));
			if (!rp || !cols || !vals) drv_die("host allocation failed");
			if (cas_csr_read_bin(bin, &nr, &nc, rp, cols, vals) == bnnz) {
				memset(M, 0, sizeof(*M));
				M->num_row = nr;
				M->num_col = nc;
				M->num_nnz = bnnz;
				M->row_ptrs = rp;
				M->cols = cols;
				M->rats = vals;
				M->col_bytes = 4;
				M->val_type = CAS_VAL_F64;
				return;
			}
			free(rp);
			free(cols);
			free(vals);
		}
	}
	const int64_t nnz = cas_mtx_read(path, &nr, &nc, NULL, NULL, NULL);
	if (nnz < 0) {
		fprintf(stderr, "Error opening or parsing %s\n", path);
		exit(1);
	}
	int64_t *rp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nr + 1));
	int32_t *cols = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
	double *vals = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
	if (!rp || !cols || !vals) drv_die("host allocation failed");
	if (cas_mtx_read(path, &nr, &nc, rp, cols, vals) != nnz) drv_die("MatrixMarket reread failed");
	if (cache && cas_csr_write_bin(bin, nr, nc, rp, cols, vals) != 0)
		fprintf(stderr, "warning: could not write the CSR cache %s\n", bin);
	memset(M, 0, sizeof(*M));
	M->num_row = nr;
	M->num_col = nc;
	M->num_nnz = nnz;
	M->row_ptrs = rp;
	M->cols = cols;
	M->rats = vals;
	M->col_bytes = 4;
	M->val_type = CAS_VAL_F64;
}

/* Device copy of a host CSR (int32 columns, fp64 values). */
static void drv_upload(const cas_csr *H, cas_csr *D) {
	*D = *H;
	void *rp = NULL, *cols = NULL, *vals = NULL;
	const size_t n = (size_t)(H->num_nnz > 0 ? H->num_nnz : 1);
	if (cudaMalloc(&rp, sizeof(int64_t) * (size_t)(H->num_row + 1)) != cudaSuccess ||
	    cudaMalloc(&cols, sizeof(int32_t) * n) != cudaSuccess || cudaMalloc(&vals, sizeof(double) * n) != cudaSuccess)
		drv_die("device allocation of the inputs failed");
	if (cudaMemcpy(rp, H->row_ptrs, sizeof(int64_t) * (size_t)(H->num_row + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(cols, H->cols, sizeof(int32_t) * (size_t)H->num_nnz, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(vals, H->rats, sizeof(double) * (size_t)H->num_nnz, cudaMemcpyHostToDevice) != cudaSuccess)
		drv_die("copy of the inputs to the device failed");
	D->row_ptrs = (int64_t *)rp;
	D->cols = cols;
	D->rats = vals;
	D->on_device = 1;
	D->owned = 0;
}

/* The HBM bandwidth for hbm_frac: CAS_PEAK_GBS, else "hbm_gbs" of the JSON
 * file CAS_PEAKS_JSON (default ./MEASURED_PEAKS.json), else 6650 GB/s. */
static double drv_peak_gbs(void) {
	const double env = drv_env_double("CAS_PEAK_GBS", 0.0);
	if (env > 0) return env;
	const char *path = getenv("CAS_PEAKS_JSON");
	FILE *f = fopen((path && *path) ? path : "MEASURED_PEAKS.json", "r");
	double v = 0.0;
	if (f) {
		char buf[8192];
		const size_t n = fread(buf, 1, sizeof(buf) - 1, f);
		fclose(f);
		buf[n] = 0;
		const char *k = strstr(buf, "\"hbm_gbs\"");
		if (k && (k = strchr(k, ':'))) v = strtod(k + 1, NULL);
	}
	return v > 0 ? v : 6650.0;
}

/* Per-driver settings of the reference's R-MAT run script (scripts/ams_rmat_run.sh:25-36). */
typedef struct {
	int high_of_64;
	double prt;
	long smt_symb, smt_numc;
} drv_script_cfg;

static drv_script_cfg drv_script(cas_accum acc) {
	if (acc == CAS_ACC_HASH) return (drv_script_cfg){16, 0.90, 11000000L, 2500000L};
	return (drv_script_cfg){22, 0.85, 7000000L, 2100000L};
}

static void drv_cfg_print(const char *driver, cas_accum acc, int device, const struct cudaDeviceProp *prop,
                          int run_num, double acc_thres) {
	const drv_script_cfg sc = drv_script(acc);
	const long threads = (long)prop->multiProcessorCount * prop->maxThreadsPerMultiProcessor;
	printf("CONFIGURATION:");
	printf("\tHASH_CONSTANT: %ld", 2654435761L);
	printf("\tTHREAD_NUM: %ld", threads);
	printf("\tAMS_HIGH_THREAD_NUM: %ld", threads * sc.high_of_64 / 64);
	printf("\tAMS_SIZE: %ld", 524288L);
	printf("\tAMS_MIN_NUM: %ld", 32768L);
	printf("\tAMS_PRT: %.6f", sc.prt);
	printf("\tAMS_DNR");
	printf("\tAMS_ACC_THRES: %.6f", acc == CAS_ACC_HYBACC ? acc_thres : 5.0);
	printf("\tSMTACT");
	printf("\tSMTACT_REAR");
	printf("\tSMTACT_QUANTILE: %.6f", 0.99);
	printf("\tSMTACT_SYMB_THRES: %ld", sc.smt_symb);
	printf("\tSMTACT_NUMC_THRES: %ld", sc.smt_numc);
	printf("\tDN_MIN: %ld", 256L);
	printf("\tGUD_ALPHA: %.6f", 0.5);
	printf("\tGUD_MIN: %ld", 256L);
	printf("\tHYB_THRES: %.6f", 0.95);
	printf("\tDRIVER: %s", driver);
	printf("\tDEVICE: %s", prop->name);
	printf("\tCUDA_DEVICE: %d", device);
	printf("\tSM_COUNT: %d", prop->multiProcessorCount);
	printf("\tRUN_NUM: %d", run_num);
	printf("\n");
}

static int cas_driver_main(int argc, char **argv, cas_accum acc, const char *driver) {
	if (argc != 2) {
		fprintf(stderr, "usage: %s <dataset>\n", argv[0]);
		return 1;
	}
	const char *dataset = argv[1];
	const char *dir = getenv("CAS_DATASET_DIR");
	if (!dir || !*dir) dir = "./dataset";
	const int run_num = (int)drv_env_long("CAS_RUN_NUM", 10);
	const int device = (int)drv_env_long("CAS_DEVICE", 0);
	const int verify = (int)drv_env_long("CAS_VERIFY", 0);
	const double acc_thres = drv_env_double("CAS_ACC_THRES", 2.0);
	const double peak_gbs = drv_peak_gbs();
	if (run_num < 2) drv_die("CAS_RUN_NUM must include a warm-up and at least one measured run");

	char org[CAS_DRIVER_PATH_LEN], trs[CAS_DRIVER_PATH_LEN];
	snprintf(org, sizeof(org), "%s/%s.org.mtx", dir, dataset);
	snprintf(trs, sizeof(trs), "%s/%s.trs.mtx", dir, dataset);

	struct cudaDeviceProp prop;
	if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess)
		drv_die("no usable CUDA device");
	drv_cfg_print(driver, acc, device, &prop, run_num, acc_thres);

	cas_csr hA, hB, dA, dB;
	/* B from <dataset>.trs.mtx as the reference's drivers read it, or, when
	 * that file is absent or CAS_TRANSPOSE is 1, B = A^T made on the device
	 * (cas_csr_transpose; the same matrix trpl_transpose writes to the file) */
	FILE *trs_f = fopen(trs, "r");
	const int gpu_trs = drv_env_long("CAS_TRANSPOSE", 0) == 1 || !trs_f;
	if (trs_f) fclose(trs_f);
	drv_load(org, &hA);
	if (!gpu_trs) {
		drv_load(trs, &hB);
		if (hA.num_col != hB.num_row) drv_die("A's columns do not match B's rows");
	}
	drv_upload(&hA, &dA);

	cas_ctx *ctx = NULL;
	if (cas_create(device, &ctx) != CAS_OK) drv_die("cas_create failed");
	if (acc == CAS_ACC_HYBACC && cas_set_acc_thres(ctx, acc_thres) != CAS_OK) drv_die(cas_last_error(ctx));
	if (gpu_trs) {
		memset(&dB, 0, sizeof(dB));
		dB.on_device = 1;
		if (cas_csr_transpose(ctx, &dA, &dB) != CAS_OK) drv_die(cas_last_error(ctx));
		memset(&hB, 0, sizeof(hB));  /* B's row pointers on the host, for flop_cnt */
		hB.num_row = dB.num_row;
		hB.num_col = dB.num_col;
		hB.num_nnz = dB.num_nnz;
		hB.row_ptrs = (int64_t *)malloc(sizeof(int64_t) * (size_t)(dB.num_row + 1));
		if (!hB.row_ptrs ||
		    cudaMemcpy(hB.row_ptrs, dB.row_ptrs, sizeof(int64_t) * (size_t)(dB.num_row + 1), cudaMemcpyDeviceToHost) !=
		        cudaSuccess)
			drv_die("copy of B's row pointers failed");
		fprintf(stderr, "%s not read: B = A^T made on the device\n", trs);
	} else {
		drv_upload(&hB, &dB);
	}

	cas_runtime sum = {0, 0, 0, 0, 0};
	int64_t nnz_c = 0;
	for (int idx = 0; idx < run_num; ++idx) {
		cas_csr C;
		memset(&C, 0, sizeof(C));
		C.on_device = 1;
		cas_runtime rt;
		const cas_status st = cas_spgemm(ctx, acc, &dA, &dB, &C, &rt);
		if (st != CAS_OK) {
			fprintf(stderr, "cas_spgemm failed (%d): %s\n", (int)st, cas_last_error(ctx));
			return 1;
		}
		nnz_c = C.num_nnz;
		if (verify && idx > 0) {
			int32_t *cols = (int32_t *)malloc(sizeof(int32_t) * (size_t)(C.num_nnz > 0 ? C.num_nnz : 1));
			double *vals = (double *)malloc(sizeof(double) * (size_t)(C.num_nnz > 0 ? C.num_nnz : 1));
			if (!cols || !vals) drv_die("host allocation failed");
			if (cudaMemcpy(cols, C.cols, sizeof(int32_t) * (size_t)C.num_nnz, cudaMemcpyDeviceToHost) != cudaSuccess ||
			    cudaMemcpy(vals, C.rats, sizeof(double) * (size_t)C.num_nnz, cudaMemcpyDeviceToHost) != cudaSuccess)
				drv_die("copy of C to the host failed");
			int64_t sum_col = 0;
			double sum_rat = 0.0;
			for (int64_t j = 0; j < C.num_nnz; ++j) {
				sum_col += cols[j];
				sum_rat += vals[j];
			}
			printf("VERIFYRESULT:\t%ld\t%ld\t%f\n", (long)C.num_nnz, (long)sum_col, sum_rat);
			free(cols);
			free(vals);
		}
		cas_csr_free(ctx, &C);
		if (idx > 0) {
			sum.init_time += rt.init_time;
			sum.symb_time += rt.symb_time;
			sum.mgmt_time += rt.mgmt_time;
			sum.numc_time += rt.numc_time;
			sum.total_time += rt.total_time;
		}
		drv_cyan();
		printf("%dth run\tinit_time: %.9f\tsymb_time: %.9f\tmgmt_time: %.9f\tnumc_time: %.9f\ttotal_time: %.9f\n", idx,
		       rt.init_time, rt.symb_time, rt.mgmt_time, rt.numc_time, rt.total_time);
		drv_reset();
		printf("\n");
	}

	/* flop_cnt outside the timed phases, as get_intprod (src/mm/mm_utils.c:981-1055) */
	const int64_t flop = cas_intprod_host(hA.num_row, hA.row_ptrs, (const int32_t *)hA.cols, hB.row_ptrs);
	const int trials = run_num - 1;
	const double tot = sum.total_time / trials, numc = sum.numc_time / trials;
	const double bytes = 12.0 * (double)hA.num_nnz + 12.0 * (double)flop + 12.0 * (double)nnz_c +
	                     16.0 * (double)(hA.num_row + 1);
	drv_green();
	printf("dataset: %s\tnum_trials: %d\tthread_num: %d\tnuma_mask: %ld\t"
	       "init_time: %.9f\tsymb_time: %.9f\tmgmt_time: %.9f\tnumc_time: %.9f\ttotal_time: %.9f\t"
	       "flop_cnt: %ld\tnumc_perf: %.9f\tperf: %.9f\t"
	       "gflops: %.3f\thbm_frac: %.4f\tdevice: %s\thbm_peak_gbs: %.1f\n",
	       dataset, trials, prop.multiProcessorCount, 1L << device, sum.init_time / trials, sum.symb_time / trials,
	       sum.mgmt_time / trials, numc, tot, (long)flop, flop / numc, flop / tot, 2.0 * flop / tot / 1e9,
	       bytes / tot / (peak_gbs * 1e9), prop.name, peak_gbs);
	drv_reset();

	if (gpu_trs) {
		cas_csr_free(ctx, &dB);
	} else {
		cudaFree((void *)dB.row_ptrs);
		cudaFree(dB.cols);
		cudaFree(dB.rats);
	}
	cas_destroy(ctx);
	cudaFree((void *)dA.row_ptrs);
	cudaFree(dA.cols);
	cudaFree(dA.rats);
	free(hA.row_ptrs);
	free(hA.cols);
	free(hA.rats);
	free(hB.row_ptrs);
	free(hB.cols);
	free(hB.rats);
	return 0;
}

#endif
