/* pdlp_oracle.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, serial FP64 restatement of the reference solver's PDLP path, used
 * by tests/ and by the CPU-baseline leg of bench.py as the checker. Nothing in
 * the product links or calls it. Each function names the reference file:line
 * it restates. Matrices are CSR with int32 indices; all vectors are double.
 */
#ifndef PDLP_ORACLE_H
#define PDLP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* COO -> CSR with the reference's stable fill order (include/sparse.hpp:24-40).
 * indptr has rows+1 entries. Pass transpose=1 for CSR(A^T) (sparse.hpp:43-50). */
void or_coo_to_csr(int rows, int cols, int64_t nnz, const int32_t* row, const int32_t* col, const double* val,
                   int transpose, int32_t* indptr, int32_t* indices, double* data);

/* y = M x over a CSR (include/sparse.hpp:52-59), left-to-right per row. */
void or_matvec(int rows, const int32_t* indptr, const int32_t* indices, const double* data, const double* x,
               double* y);

/* Independent KKT check (src/verify.cpp:24-103). out[0..6] = eps_P, eps_D,
 * eps_G, objective (c'x + offset), dual objective (+ offset), max row
 * violation, max bound violation. */
void or_verify(int m, int n, const int32_t* a_ptr, const int32_t* a_idx, const double* a_val,
               const int32_t* at_ptr, const int32_t* at_idx, const double* at_val, const double* c,
               const double* rL, const double* rU, const double* l, const double* u, double obj_offset,
               const double* x, const double* y, double* out);

/* Ruiz (ruiz_passes) + Pock-Chambolle alpha=1 scaling of an LP (src/scaling.cpp:25-84,
 * LP case: no integer columns, no Q). Outputs are the scaled values in COO order,
 * the scaled c, rL, rU, l, u and the scalings Dr (m) and Dc (n). */
void or_scale(int m, int n, int64_t nnz, const int32_t* row, const int32_t* col, const double* val,
              const double* c, const double* rL, const double* rU, const double* l, const double* u,
              int ruiz_passes, double* val_s, double* c_s, double* rL_s, double* rU_s, double* l_s,
              double* u_s, double* Dr, double* Dc);

/* One LP in the form pdlp_run receives it (include/pdlp_algo.hpp:50-52). */
typedef struct {
    int m, n;
    int64_t nnz;
    const int32_t* row;
    const int32_t* col;
    const double* val;
    const double *c, *rL, *rU, *l, *u;
    double obj_offset;
} or_lp;

/* Restarted PDLP with the reference's CPU backend semantics
 * (include/pdlp_algo.hpp:49-185 + src/pdlp.cpp:97-142), FP64, serial.
 * x (n) and y (m) receive the returned point in unscaled PDLP-form space.
 * info[0] = iterations (attempts), info[1] = restarts, info[2] = converged,
 * info[3] = accepted steps. eps[0..2] = eps_P, eps_D, eps_G.
 * If trace is not NULL it receives, per attempt k < trace_len, the step size
 * eta used by that attempt (negated when the attempt was rejected). */
int or_pdlp_run(const or_lp* unscaled, const or_lp* scaled, const double* Dr, const double* Dc,
                int max_iterations, int check_every, double tol, double* x, double* y, int* info, double* eps,
                double* trace, int trace_len);

/* The benchmark LP generators, restated from the product's seeded generators
 * so that reference-side runs build the same LPs without the product library.
 * Random equality LP: k distinct rows per column, values U[-1,1] (optionally
 * rounded to FP32), b = A x0, c = A^T y0 + z0, 0 <= x <= 10; COO of n*k entries
 * in column order. Transportation LP: S sources x D sinks, 2 unit entries per
 * arc, integer supplies and demands, integer costs, 0 <= x. Return 0, or 1 on
 * bad sizes. */
int or_gen_random_lp(int m, int n, int k, uint64_t seed, int fp32_values, int32_t* row, int32_t* col, double* val,
                     double* c, double* rL, double* rU, double* l, double* u);
int or_gen_transport(int S, int D, uint64_t seed, int32_t* row, int32_t* col, double* val, double* c, double* rL,
                     double* rU, double* l, double* u);

#ifdef __cplusplus
}
#endif
#endif
