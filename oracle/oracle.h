/* ORACLE — test infrastructure only.
 *
 * CPU restatement of the reference's algorithms on the FDMT + search hot path.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
 * it, and only as the checker.  The product (cpp_projects_b200/) never links
 * or calls anything here.
 *
 * Parity pinning: the FDMT restatement is checked bit-for-bit against the
 * reference's own CFdmtCpu compiled from its sources (oracle/_ref, built by
 * oracle/Makefile) and the search restatement against the reference's golden
 * CSVs (clusterization_forpravir/Candidates{1,2}.csv, copied as fixtures under
 * tests/golden/).
 */
#ifndef BFS_ORACLE_H
#define BFS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same 16-byte layout as the reference's Cand (Clusterization/Candidate.cuh:4-10). */
typedef struct orc_cand { int mt; int mdt; int mwidth; float msnr; } orc_cand;

/* --- FDMT (reference: MyVSLib_C++/FDMT/FdmtB.cpp, FdmtCpu.cpp) --------- */
int orc_fdmt_niter(int nchan);
/* rows_per_level[0..niter] = total rows of each level's plane; returns niter or <0 */
int orc_fdmt_rows(float fmin, float fmax, int nchan, int max_dt, int* rows_per_level, int cap);
/* Row tables of level `level` (>=1): for each output row, the tail row, the
 * head row (-1 for a copied row) and the head shift.  Returns the row count. */
int orc_fdmt_tables(float fmin, float fmax, int nchan, int max_dt, int level,
                    int* a_row, int* b_row, int* shift, int cap);
int orc_fdmt_run_f32(float fmin, float fmax, int nchan, int cols, int max_dt,
                     const float* in, float* out, int b_ones);
int orc_fdmt_run_f64(float fmin, float fmax, int nchan, int cols, int max_dt,
                     const double* in, double* out, int b_ones);
/* The FP32 FDMT with the planes of levels kstore..niter-1 rounded as a
 * 16-bit store would round them (prec ORC_PREC_F16 / ORC_PREC_BF16), row g
 * scaled by 2^-ceil(log2(channels summed into g)) first; levels below kstore
 * (a fused head's shared-memory levels) stay FP32. */
enum { ORC_PREC_F16 = 1, ORC_PREC_BF16 = 2 };
int orc_fdmt_run_lowp(float fmin, float fmax, int nchan, int cols, int max_dt,
                      const float* in, float* out, int b_ones, int prec, int kstore);
/* out[i] = in[i] rounded to the nearest binary16 / bfloat16 (ties to even). */
void orc_round16(const float* in, float* out, int64_t n, int prec);
/* Adjoint (transpose) of the FDMT: gx (nchan x cols) = F^T gy (max_dt x cols);
 * the FP32 version sums in the product's fixed order. */
int orc_fdmt_adjoint_f32(float fmin, float fmax, int nchan, int cols, int max_dt,
                         const float* gy, float* gx);
int orc_fdmt_adjoint_f64(float fmin, float fmax, int nchan, int cols, int max_dt,
                         const double* gy, double* gx);

/* --- Pravir-plan FDMT (reference: MyVSLib_C++/FDMT_PRAVIR/) -------------
 * All return < 0 where the reference throws.  rows_per_level[0..niter];
 * orc_pravir_level: sub-band row cumsum (nsub+1), dt of every row and, for
 * level >= 1, tail row, head row (-1: copied) and offset; returns the rows. */
int orc_pravir_rows(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,
                    long dt_min, int* rows_per_level, int cap);
int orc_pravir_level(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,
                     long dt_min, int level, int* cum, int* dt, int* a_row, int* b_row, int* shift,
                     int cap);
int orc_pravir_run_f32(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,
                       long dt_min, const float* in, float* out);
int orc_pravir_run_f64(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,
                       long dt_min, const double* in, double* out);
int orc_pravir_adjoint_f32(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,
                           long dt_min, const float* gy, float* gx);
int orc_pravir_adjoint_f64(float fmin, float fmax, int nchans, int nsamps, long dt_max, long dt_step,
                           long dt_min, const double* gy, double* gx);

/* --- search (reference: MyVSLib_C++/Clusterization/ sources) --------------- */
int64_t orc_boxcar(const float* plane, int rows, int cols, float thr, int mode,
                   int param, orc_cand* out, int64_t cap);
int64_t orc_boxcar_mt(const float* plane, int rows, int cols, float thr, int mode,
                      int param, orc_cand* out, int64_t cap);
void orc_norm_rows(const float* in, float* out, int rows, int cols,
                   float* mean_out, float* std_out);
int orc_select_delegates(const orc_cand* c, const int* perm, const int* offsets,
                         int ngroups, int block, int* delegates);
int orc_cluster(const orc_cand* c, int n, const int* metrics, int* perm_out,
                int* offsets_out, int* delegates_out);
void orc_calc_fdmt_inputs(float* inout, int rows, int cols, float* norm_input,
                          float* stats_out);

#ifdef __cplusplus
}
#endif
#endif
