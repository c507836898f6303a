/*
 * ORACLE -- test infrastructure only. Nothing in the product (tccg_b200/)
 * links or calls this file; tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg use it as the checker.
 *
 * A C restatement of the loop nest that TCCG emits as its correctness
 * reference, `referenceVersion` (tccg/tccg.py:686-723):
 *
 *   for every index of C, the LAST index of C outermost, the first innermost
 *   (tccg.py:696 iterates C.indices[::-1]);
 *     tmp = 0 (in the tensor's float type, tccg.py:702)
 *     for every contracted index, in getContractedIndices order
 *       (tccg/tccg_util.py:597-611), the first one outermost (tccg.py:705-708)
 *       tmp += A[...] * B[...]                                   (tccg.py:710)
 *     C[...] = alpha * tmp             if beta == 0              (tccg.py:714)
 *     C[...] = alpha * tmp + beta * C  otherwise                 (tccg.py:716)
 *
 * Extents and strides are runtime arguments here (TCCG bakes them in), and a
 * half-open range [c_begin, c_end) of C's column-major linear index selects a
 * slab of the loop nest (the loop order above visits C in exactly that linear
 * order), which lets large contractions be timed or checked on a bounded
 * sample. OpenMP splits the slab across threads like the reference's
 * `#pragma omp parallel for collapse(...)` when threads > 1 (tccg.py:694-695).
 *
 * Build: see oracle/Makefile (gcc -O3 -fopenmp -shared -fPIC).
 */
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_MAX_MODES 16

/* One C element: decode the column-major linear index into C's modes. */
static inline void decode_c(int64_t lin, int nc, const int64_t* ext, int64_t* idx) {
  for (int d = 0; d < nc; ++d) {
    idx[d] = lin % ext[d];
    lin /= ext[d];
  }
}

#define DEFINE_LOOPNEST(NAME, T, ACC)                                                   \
  int NAME(int nc, const int64_t* c_ext, const int64_t* c_str_a, const int64_t* c_str_b, \
           const int64_t* c_str_c, int nk, const int64_t* k_ext, const int64_t* k_str_a, \
           const int64_t* k_str_b, const T* A, const T* B, T* C, T alpha, T beta,       \
           int64_t c_begin, int64_t c_end, int threads) {                               \
    if (nc < 1 || nc > ORACLE_MAX_MODES || nk < 0 || nk > ORACLE_MAX_MODES) return -1;  \
    int64_t total = 1;                                                                  \
    for (int d = 0; d < nc; ++d) total *= c_ext[d];                                     \
    if (c_begin < 0) c_begin = 0;                                                       \
    if (c_end < 0 || c_end > total) c_end = total;                                      \
    int64_t ktot = 1;                                                                   \
    for (int d = 0; d < nk; ++d) ktot *= k_ext[d];                                      \
    if (threads < 1) threads = 1;                                                       \
    _Pragma("omp parallel for schedule(static) num_threads(threads)")                   \
    for (int64_t lin = c_begin; lin < c_end; ++lin) {                                   \
      int64_t ci[ORACLE_MAX_MODES];                                                     \
      decode_c(lin, nc, c_ext, ci);                                                     \
      int64_t offa = 0, offb = 0, offc = 0;                                             \
      for (int d = 0; d < nc; ++d) {                                                    \
        offa += ci[d] * c_str_a[d];                                                     \
        offb += ci[d] * c_str_b[d];                                                     \
        offc += ci[d] * c_str_c[d];                                                     \
      }                                                                                 \
      ACC tmp = 0;                                                                      \
      /* contracted loops: k_ext[0] outermost, k_ext[nk-1] innermost */                  \
      int64_t ki[ORACLE_MAX_MODES];                                                     \
      for (int d = 0; d < nk; ++d) ki[d] = 0;                                           \
      int64_t ka = 0, kb = 0;                                                           \
      for (int64_t kk = 0; kk < ktot; ++kk) {                                           \
        tmp += (ACC)A[offa + ka] * (ACC)B[offb + kb];                                   \
        for (int d = nk - 1; d >= 0; --d) { /* odometer, innermost first */            \
          ki[d]++;                                                                      \
          ka += k_str_a[d];                                                             \
          kb += k_str_b[d];                                                             \
          if (ki[d] < k_ext[d]) break;                                                  \
          ka -= ki[d] * k_str_a[d];                                                     \
          kb -= ki[d] * k_str_b[d];                                                     \
          ki[d] = 0;                                                                    \
        }                                                                               \
      }                                                                                 \
      if (beta == (T)0)                                                                 \
        C[offc] = (T)(alpha * tmp);                                                     \
      else                                                                              \
        C[offc] = (T)(alpha * tmp + beta * C[offc]);                                    \
    }                                                                                   \
    return 0;                                                                           \
  }

/* Single precision: tmp is float, as in the emitted reference for -floatType=s. */
DEFINE_LOOPNEST(oracle_loopnest_f32, float, float)
/* Double precision: tmp is double (-floatType=d). */
DEFINE_LOOPNEST(oracle_loopnest_f64, double, double)
/* Single-precision operands evaluated with a double accumulator: the FP64
 * reference used to measure errors of the FP32/BF16 paths. */
DEFINE_LOOPNEST(oracle_loopnest_f32_acc64, float, double)

/*
 * FP64 values of selected C entries: for each of `ns` column-major linear C
 * indices in `lins`, out[s] = alpha * sum_k A*B (+ beta * C[lin]) with all
 * arithmetic in double. A, B, C are float (is_double = 0) or double (1).
 */
int oracle_sample_f64(int nc, const int64_t* c_ext, const int64_t* c_str_a,
                      const int64_t* c_str_b, const int64_t* c_str_c, int nk,
                      const int64_t* k_ext, const int64_t* k_str_a, const int64_t* k_str_b,
                      const void* A, const void* B, const void* C, int is_double,
                      double alpha, double beta, int64_t ns, const int64_t* lins,
                      double* out, int threads) {
  if (nc < 1 || nc > ORACLE_MAX_MODES || nk < 0 || nk > ORACLE_MAX_MODES) return -1;
  int64_t ktot = 1;
  for (int d = 0; d < nk; ++d) ktot *= k_ext[d];
  if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
  for (int64_t s = 0; s < ns; ++s) {
    int64_t ci[ORACLE_MAX_MODES];
    decode_c(lins[s], nc, c_ext, ci);
    int64_t offa = 0, offb = 0, offc = 0;
    for (int d = 0; d < nc; ++d) {
      offa += ci[d] * c_str_a[d];
      offb += ci[d] * c_str_b[d];
      offc += ci[d] * c_str_c[d];
    }
    double tmp = 0;
    int64_t ki[ORACLE_MAX_MODES];
    for (int d = 0; d < nk; ++d) ki[d] = 0;
    int64_t ka = 0, kb = 0;
    for (int64_t kk = 0; kk < ktot; ++kk) {
      double a = is_double ? ((const double*)A)[offa + ka] : (double)((const float*)A)[offa + ka];
      double b = is_double ? ((const double*)B)[offb + kb] : (double)((const float*)B)[offb + kb];
      tmp += a * b;
      for (int d = nk - 1; d >= 0; --d) {
        ki[d]++;
        ka += k_str_a[d];
        kb += k_str_b[d];
        if (ki[d] < k_ext[d]) break;
        ka -= ki[d] * k_str_a[d];
        kb -= ki[d] * k_str_b[d];
        ki[d] = 0;
      }
    }
    double r = alpha * tmp;
    if (beta != 0.0) {
      double c = is_double ? ((const double*)C)[offc] : (double)((const float*)C)[offc];
      r += beta * c;
    }
    out[s] = r;
  }
  return 0;
}

/* TCCG's deterministic inputs (tccg.py:957-971), written as floats the way
 * the emitted main.cpp does: ((float)(10 + ((i+o)*m) % 100)) / 110.0.
 * which = 0: A (o=1, m=17); 1: B (o=2, m=3); 2: C (o=3, m=13). */
int oracle_tccg_init_f32(int which, float* x, int64_t n) {
  int64_t o, m;
  if (which == 0) { o = 1; m = 17; }
  else if (which == 1) { o = 2; m = 3; }
  else if (which == 2) { o = 3; m = 13; }
  else return -1;
  for (int64_t i = 0; i < n; ++i) x[i] = (float)((float)(10 + ((i + o) * m) % 100) / 110.0);
  return 0;
}

int oracle_tccg_init_f64(int which, double* x, int64_t n) {
  int64_t o, m;
  if (which == 0) { o = 1; m = 17; }
  else if (which == 1) { o = 2; m = 3; }
  else if (which == 2) { o = 3; m = 13; }
  else return -1;
  for (int64_t i = 0; i < n; ++i) x[i] = (double)((float)(10 + ((i + o) * m) % 100) / 110.0);
  return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
