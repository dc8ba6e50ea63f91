/*
 * TEST INFRASTRUCTURE — not part of the product.
 *
 * Direct-call harness around the reference's own CPU SpGEMM kernels
 * (fukien/contention-aware-spgemm).  It is compiled together with the
 * unmodified reference sources src/inc/utils.c, src/mm/mm_utils.c and
 * src/ams/ams_utils.c (see oracle/Makefile) into oracle/_ref/libref_<algo>.so,
 * one library per accumulator because every tuning knob of the reference is a
 * compile-time macro.
 *
 * ref_spgemm() runs the same four timed phases, in the same order, as the
 * static driver functions it mirrors:
 *   hashspgemm()    src/ams_hashspgemm.c:36-205
 *   hserscspgemm()  src/ams_hserscspgemm.c:36-210
 *   hybaccspgemm()  src/ams_hybaccspgemm.c:36-215
 * for the run-script build (-DAMS_DNR -DSMTACT -DSMTACT_REAR,
 * scripts/ams_run_common.sh:20-33).  Those functions are `static` inside the
 * driver executables, so they cannot be called from a library; this harness
 * restates their call sequence and calls the reference's exported functions.
 *
 * Two departures from the drivers, both for test use:
 *  * the harness returns C instead of freeing it (the drivers free it at the
 *    end of every run, src/ams_hashspgemm.c:343), and
 *  * it refuses inputs for which pack_ams_pack() would compute zero morsels:
 *    the reference then calls mmap(0) and exit(1)
 *    (src/ams/ams_utils.c:1418-1425, src/inc/utils.c:204-209).  ref_spgemm()
 *    returns 1 in that case instead of taking the calling process down.
 */
#include "ams/ams_utils.h"

#ifndef CAS_REF_ALGO
#error "define CAS_REF_ALGO: 0 = hash, 1 = hsersc, 2 = hybacc"
#endif

extern numa_cfg_t numa_cfg;
#ifdef SMTACT
extern my_cnt_t cph_mf_th;
extern bool ht_dis_flag;
#endif

static int g_ref_ready = 0;

/* NUMA setup of main() (src/ams_hashspgemm.c:232-265), reduced to the single
 * node the shim reports. */
static void ref_setup(void) {
	if (g_ref_ready) {
		return;
	}
	numa_cfg_init(&numa_cfg);
	numa_cfg.node_idx = 0;
	numa_bitmask_clearall(numa_cfg.numa_mask);
	numa_bitmask_setbit(numa_cfg.numa_mask, 0);
	g_ref_ready = 1;
}

int ref_algo(void) { return CAS_REF_ALGO; }
int ref_thread_num(void) { return THREAD_NUM; }
long ref_morsel_size(void) { return (long) MIN(AMS_MIN_NUM, AMS_SIZE / sizeof(my_cnt_t)); }
double ref_acc_thres(void) { return AMS_ACC_THRES; }

/* Total intermediate products, the reference's flop_cnt log field
 * (get_intprod, src/mm/mm_utils.c:1023-1055). */
long ref_intprod(csr_t *A, csr_t *B) {
	ref_setup();
	my_cnt_t *row = (my_cnt_t *) malloc(sizeof(my_cnt_t) * (A->num_row > 0 ? A->num_row : 1));
	my_cnt_t p = get_intprod(A, B, row);
	free(row);
	return (long) p;
}

/* The reference's MatrixMarket loader (raw2csr -> mtx2csr -> mtx2trpl ->
 * trpl2csr, src/mm/mm_utils.c:451-692, 730) into M; release with ref_free_csr. */
void ref_load_mtx(const char *path, csr_t *M) {
	ref_setup();
	memset(M, 0, sizeof(csr_t));
	raw2csr(M, path, &numa_cfg);
}

void ref_free_csr(csr_t *C) {
	if (C->row_ptrs) {
		free_csr(C);
	}
	memset(C, 0, sizeof(csr_t));
}

/* Returns 0 and fills C (allocated by the reference's alloc2_memory; release
 * with ref_free_csr) and rt; returns 1 when an input is below one morsel. */
int ref_spgemm(csr_t *csr_a, csr_t *csr_b, csr_t *csr_c, runtime_t *rt) {
	ref_setup();
	numa_cfg_t *ncfg = &numa_cfg;
	const my_cnt_t morsel = MIN(AMS_MIN_NUM, AMS_SIZE / sizeof(my_cnt_t));
	struct timespec t0, t1;
	runtime_t runtime;
	memset(csr_c, 0, sizeof(csr_t));
	if (csr_a->num_nnz < morsel || csr_a->num_row < 1) {
		return 1;
	}

	/* INIT */
	clock_gettime(CLOCK_REALTIME, &t0);
	csr_c->num_row = csr_a->num_row;
	csr_c->num_col = csr_b->num_col;
	csr_c->row_ptrs = (my_cnt_t *) alloc2_memory(sizeof(my_cnt_t) * (csr_c->num_row + 1), ncfg);
	memset(csr_c->row_ptrs, 0, sizeof(my_cnt_t) * (csr_c->num_row + 1));
	ams_pack_t ams_pack;
	memset(&ams_pack, 0, sizeof(ams_pack_t));
	ams_bin_t ams_bin;
	init_ams_bin(&ams_bin, &ams_pack, csr_a, ncfg);
	my_cnt_t max_row_flp = 0;
	flp_populate(csr_a, csr_b, ams_bin.row_flp);
	scan(ams_bin.ps_row_flp, ams_bin.row_flp, csr_a->num_row + 1);
#ifdef SMTACT
	ht_dis_flag = false;
	cph_mf_th = SMTACT_SYMB_THRES;
	max_row_flp = pack_ams_pack(csr_a->row_ptrs, &ams_bin, ncfg);
#endif
	clock_gettime(CLOCK_REALTIME, &t1);
	runtime.init_time = diff_sec(t0, t1);

	/* SYMBOLIC */
	clock_gettime(CLOCK_REALTIME, &t0);
	size_t ht_len = sizeof(my_cnt_t) * THREAD_NUM * NEXT_POW_2(csr_c->num_col);
	my_cnt_t *ht_check = (my_cnt_t *) alloc2_memory(ht_len, ncfg);
	ams_hash_symb_dnr(csr_a, csr_b, ht_check, &ams_bin);
	scan(csr_c->row_ptrs, ams_bin.row_nz, csr_a->num_row + 1);
	csr_c->num_nnz = csr_c->row_ptrs[csr_c->num_row];
	clock_gettime(CLOCK_REALTIME, &t1);
	runtime.symb_time = diff_sec(t0, t1);
#if CAS_REF_ALGO == 1
	dealloc_memory(ht_check, ht_len);
	ht_check = NULL;
#endif

	if (csr_c->num_nnz < morsel) {
		/* pack_ams_pack(C.row_ptrs) below would exit(1) */
		if (ht_check) {
			dealloc_memory(ht_check, ht_len);
		}
		free_ams_pack(&ams_pack);
		free_ams_bin(&ams_bin);
		dealloc_memory(csr_c->row_ptrs, sizeof(my_cnt_t) * (csr_c->num_row + 1));
		memset(csr_c, 0, sizeof(csr_t));
		return 1;
	}

	/* MANAGEMENT */
	clock_gettime(CLOCK_REALTIME, &t0);
	csr_c->cols = (my_cnt_t *) alloc2_memory(sizeof(my_cnt_t) * csr_c->num_nnz, ncfg);
	csr_c->rats = (my_rat_t *) alloc2_memory(sizeof(my_rat_t) * csr_c->num_nnz, ncfg);
	free_ams_pack(&ams_pack);
#ifdef SMTACT
	ht_dis_flag = false;
	cph_mf_th = SMTACT_NUMC_THRES;
#endif
	max_row_flp = pack_ams_pack(csr_c->row_ptrs, &ams_bin, ncfg);
	clock_gettime(CLOCK_REALTIME, &t1);
	runtime.mgmt_time = diff_sec(t0, t1);

	/* NUMERIC */
	clock_gettime(CLOCK_REALTIME, &t0);
#if CAS_REF_ALGO == 0
	my_rat_t *ht_value = (my_rat_t *) alloc2_memory(
		sizeof(my_rat_t) * THREAD_NUM * NEXT_POW_2(csr_c->num_col), ncfg);
	ams_hash_numc(csr_a, csr_b, csr_c, ht_check, ht_value, &ams_bin);
	dealloc_memory(ht_check, ht_len);
	dealloc_memory(ht_value, sizeof(my_rat_t) * THREAD_NUM * NEXT_POW_2(csr_c->num_col));
#elif CAS_REF_ALGO == 1
	keyval_t *keyval_org = (keyval_t *) alloc2_memory(sizeof(keyval_t) * THREAD_NUM * max_row_flp, ncfg);
	keyval_t *aux = (keyval_t *) alloc2_memory(sizeof(keyval_t) * THREAD_NUM * max_row_flp, ncfg);
	ams_hsersc_numc(csr_a, csr_b, csr_c, keyval_org, aux, max_row_flp, &ams_bin);
	dealloc_memory(keyval_org, sizeof(keyval_t) * THREAD_NUM * max_row_flp);
	dealloc_memory(aux, sizeof(keyval_t) * THREAD_NUM * max_row_flp);
#else
	my_rat_t *ht_value = (my_rat_t *) alloc2_memory(
		sizeof(my_rat_t) * THREAD_NUM * NEXT_POW_2(csr_c->num_col), ncfg);
	keyval_t *keyval_org = (keyval_t *) alloc2_memory(sizeof(keyval_t) * THREAD_NUM * max_row_flp, ncfg);
	keyval_t *aux = (keyval_t *) alloc2_memory(sizeof(keyval_t) * THREAD_NUM * max_row_flp, ncfg);
	ams_hybacc_numc(csr_a, csr_b, csr_c, keyval_org, aux, max_row_flp, ht_check, ht_value, &ams_bin);
	dealloc_memory(keyval_org, sizeof(keyval_t) * THREAD_NUM * max_row_flp);
	dealloc_memory(aux, sizeof(keyval_t) * THREAD_NUM * max_row_flp);
	dealloc_memory(ht_check, ht_len);
	dealloc_memory(ht_value, sizeof(my_rat_t) * THREAD_NUM * NEXT_POW_2(csr_c->num_col));
#endif
	free_ams_pack(&ams_pack);
	free_ams_bin(&ams_bin);
	clock_gettime(CLOCK_REALTIME, &t1);
	runtime.numc_time = diff_sec(t0, t1);
	runtime.total_time = runtime.init_time + runtime.symb_time + runtime.mgmt_time + runtime.numc_time;
	if (rt) {
		*rt = runtime;
	}
	return 0;
}
