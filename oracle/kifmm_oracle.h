/*
 * TEST INFRASTRUCTURE — the oracle.  A plain-C CPU restatement of the
 * reference's exact-FP64 KIFMM evaluator (fmm/omp.cc with fmm/trans.cc's
 * scatter/gather), used only by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker.  Never linked into the product.
 *
 * Parity is pinned: tests compare this restatement with the reference itself,
 * compiled from its sources by oracle/Makefile (oracle/_ref) and run through
 * oracle/ref_harness.cc, and with golden vectors under tests/golden/.
 */
#ifndef KIFMM_ORACLE_H
#define KIFMM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int num_nodes, num_levels, num_src, num_trg;
  const int *parent, *child, *depth, *tag, *path;
  const int *src_beg, *src_num, *trg_beg, *trg_num, *src_perm, *trg_perm, *node_level;
  const int *u_ptr, *u_idx, *v_ptr, *v_idx, *w_ptr, *w_idx, *x_ptr, *x_idx;
} oracle_tree;

typedef struct {
  const double *uc2ue, *ue2uc, *dc2de, *de2dc, *ue2dc; /* layouts of kfmm_operators */
} oracle_ops;

/* Full evaluation: original-order inputs -> original-order potentials.
 * Optional per-node outputs (num_nodes * P each, may be NULL): upward
 * equivalent density, downward check potential, downward equivalent density.
 * Returns 0 on success. */
int oracle_evaluate(const oracle_tree* t, int np, const oracle_ops* ops, const double* sx,
                    const double* sy, const double* sz, const double* den, const double* tx,
                    const double* ty, const double* tz, double* pot, double* uden_out,
                    double* dchk_out, double* dden_out);

/* 0: the reference's summation order; 1: all direct sums and matrix-vector
 * products in descending order (an equally valid FP64 evaluation, used to
 * measure the algorithm's own rounding floor).  Process-wide. */
void oracle_set_order(int reverse);

/* Precision of the operator matrix-vector products: 0 FP64 (reference),
 * 1 FP32, 2 split-TF32 three-pass with FP32 accumulation.  Process-wide;
 * used to measure the sensitivity of the potentials to reduced-precision
 * level products. */
void oracle_set_product_precision(int mode);

/* ulist__direct_evaluation over all sources for selected targets (the check of
 * fmm/driver.cc:142-206 with a zeroed accumulator). */
void oracle_direct(int nt, const double* tx, const double* ty, const double* tz, int ns,
                   const double* sx, const double* sy, const double* sz, const double* den,
                   double* pot);

#ifdef __cplusplus
}
#endif

#endif
