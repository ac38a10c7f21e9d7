/*
 * TEST INFRASTRUCTURE - the CPU oracle of the transposition. Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load it; the product path never does.
 *
 * A plain-C restatement of the scalar loop nest that TTC generates as its correctness reference
 * (GPUreference.py:33-244 in the TTC project) and of its CPU baseline semantics:
 *
 *   for every index tuple (i0..iN-1) of A:
 *     B[sum_j i_{perm[j]} * strideB[j]] = alpha*A[sum_i i_i * strideA[i]] (+ beta*B[...])
 *
 *   strideA[i] = prod_{k<i} lda[k], strideB[j] = prod_{k<j} ldb[k]      (GPUreference.py:217-230)
 *
 * The update follows GPUreference.py:90-137 exactly:
 *   real A/B:    B = alpha*A + beta*B, alpha in A's precision, beta in B's (GPUreference.py:44-54),
 *                C promotion rules (float*float stays float, float+double is double)
 *   complex:     cuCmul(cuAlpha, A) [+ cuCmul(cuBeta, B) via cuCadd], with cuCmul(x, y) =
 *                (xr*yr - xi*yi, xr*yi + xi*yr) and cuComplexDoubleToFloat / FloatToDouble
 *                applied to alpha*A before the addition for the mixed pairs zc / cz.
 * The reference only accepts a real alpha/beta (cuAlpha = make_cuComplex(alpha, 0)); this oracle
 * takes the imaginary parts as well, for the complex-alpha extension.
 *
 * Build with -ffp-contract=off so no multiply-add is fused: every product and sum is rounded
 * once, as the expressions are written.
 */
#include <stdint.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OS = 0, OD = 1, OC = 2, OZ = 3 };

typedef struct { float re, im; } cfloat;
typedef struct { double re, im; } cdouble;

static inline cfloat cmulf(cfloat x, cfloat y) {
  cfloat r;
  r.re = (x.re * y.re) - (x.im * y.im);
  r.im = (x.re * y.im) + (x.im * y.re);
  return r;
}
static inline cdouble cmul(cdouble x, cdouble y) {
  cdouble r;
  r.re = (x.re * y.re) - (x.im * y.im);
  r.im = (x.re * y.im) + (x.im * y.re);
  return r;
}

/* One element update. a: pointer to the A element, b: pointer to the B element. */
static inline void update(int ta, int tb, int beta_nz, const void* a, void* b, const double* alpha,
                          const double* beta) {
  if (ta == OS && tb == OS) {
    const float al = (float)alpha[0];
    float x = *(const float*)a;
    if (beta_nz) {
      const float be = (float)beta[0];
      *(float*)b = al * x + be * *(float*)b;
    } else {
      *(float*)b = al * x;
    }
  } else if (ta == OD && tb == OD) {
    const double al = alpha[0];
    double x = *(const double*)a;
    if (beta_nz)
      *(double*)b = al * x + beta[0] * *(double*)b;
    else
      *(double*)b = al * x;
  } else if (ta == OS && tb == OD) {
    const float al = (float)alpha[0];
    float x = *(const float*)a;
    if (beta_nz)
      *(double*)b = al * x + beta[0] * *(double*)b; /* float product, promoted */
    else
      *(double*)b = al * x;
  } else if (ta == OD && tb == OS) {
    const double al = alpha[0];
    double x = *(const double*)a;
    if (beta_nz) {
      const float be = (float)beta[0];
      *(float*)b = (float)(al * x + be * *(float*)b); /* float product, double sum */
    } else {
      *(float*)b = (float)(al * x);
    }
  } else if (ta == OC && tb == OC) {
    cfloat al = {(float)alpha[0], (float)alpha[1]};
    cfloat t = cmulf(al, *(const cfloat*)a);
    if (beta_nz) {
      cfloat be = {(float)beta[0], (float)beta[1]};
      cfloat u = cmulf(be, *(cfloat*)b);
      t.re = t.re + u.re;
      t.im = t.im + u.im;
    }
    *(cfloat*)b = t;
  } else if (ta == OZ && tb == OZ) {
    cdouble al = {alpha[0], alpha[1]};
    cdouble t = cmul(al, *(const cdouble*)a);
    if (beta_nz) {
      cdouble be = {beta[0], beta[1]};
      cdouble u = cmul(be, *(cdouble*)b);
      t.re = t.re + u.re;
      t.im = t.im + u.im;
    }
    *(cdouble*)b = t;
  } else if (ta == OC && tb == OZ) {
    cfloat al = {(float)alpha[0], (float)alpha[1]};
    cfloat t = cmulf(al, *(const cfloat*)a);
    cdouble r = {(double)t.re, (double)t.im};
    if (beta_nz) {
      cdouble be = {beta[0], beta[1]};
      cdouble u = cmul(be, *(cdouble*)b);
      r.re = r.re + u.re;
      r.im = r.im + u.im;
    }
    *(cdouble*)b = r;
  } else if (ta == OZ && tb == OC) {
    cdouble al = {alpha[0], alpha[1]};
    cdouble t = cmul(al, *(const cdouble*)a);
    cfloat r = {(float)t.re, (float)t.im};
    if (beta_nz) {
      cfloat be = {(float)beta[0], (float)beta[1]};
      cfloat u = cmulf(be, *(cfloat*)b);
      r.re = r.re + u.re;
      r.im = r.im + u.im;
    }
    *(cfloat*)b = r;
  }
}

static int esize(int t) { return t == OS ? 4 : (t == OZ ? 16 : 8); }

/* Argument checks of ttc.py:733-768: perm is a permutation, lda[i] >= size[i], ldb[j] >= size[perm[j]]. */
static int check_args(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb) {
  int seen[16] = {0}, i;
  for (i = 0; i < rank; ++i) {
    if (perm[i] < 0 || perm[i] >= rank || seen[perm[i]]) return -1;
    seen[perm[i]] = 1;
    if (size[i] < 0) return -1;
    if (lda && lda[i] < size[i]) return -1;
    if (ldb && ldb[i] < size[perm[i]]) return -1;
  }
  return 0;
}

/*
 * Returns 0 on success, -1 on invalid arguments. size/lda/ldb/perm follow TTC's conventions;
 * lda/ldb may be NULL (dense). alpha/beta point to {re, im} pairs (im ignored for real types).
 * The loop order does not change the result: every B element is written exactly once.
 */
int ttco_transpose(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb,
                   int type_a, int type_b, const double* alpha, const double* beta, int beta_nonzero,
                   const void* A, void* B) {
  int64_t sA[16], sBpos[16], sB[16], idx[16];
  int i, j;
  if (rank < 1 || rank > 16 || check_args(rank, perm, size, lda, ldb)) return -1;
  sA[0] = 1;
  sBpos[0] = 1;
  for (i = 1; i < rank; ++i) {
    sA[i] = sA[i - 1] * (lda ? lda[i - 1] : size[i - 1]);
    sBpos[i] = sBpos[i - 1] * (ldb ? ldb[i - 1] : size[perm[i - 1]]);
  }
  for (j = 0; j < rank; ++j) sB[perm[j]] = sBpos[j];
  for (i = 0; i < rank; ++i) {
    if (size[i] == 0) return 0;
    idx[i] = 0;
  }
  const int ea = esize(type_a), eb = esize(type_b);
  const char* a = (const char*)A;
  char* b = (char*)B;
  for (;;) {
    int64_t oa = 0, ob = 0;
    for (i = 0; i < rank; ++i) {
      oa += idx[i] * sA[i];
      ob += idx[i] * sB[i];
    }
    update(type_a, type_b, beta_nonzero, a + oa * ea, b + ob * eb, alpha, beta);
    for (i = 0; i < rank; ++i) {
      if (++idx[i] < size[i]) break;
      idx[i] = 0;
    }
    if (i == rank) break;
  }
  return 0;
}

/*
 * Multi-threaded form of the same loop nest, as TTC's generated reference is OpenMP-parallel over
 * all but the innermost loop (GPUreference.py:210, "#pragma omp parallel for collapse(d-1)").
 * Dimension 0 is the inner loop; the other dimensions are flattened and split across threads.
 */
int ttco_transpose_par(int rank, const int* perm, const int64_t* size, const int64_t* lda, const int64_t* ldb,
                       int type_a, int type_b, const double* alpha, const double* beta, int beta_nonzero,
                       const void* A, void* B, int nthreads) {
  int64_t sA[16], sBpos[16], sB[16];
  int i, j;
  if (rank < 1 || rank > 16 || check_args(rank, perm, size, lda, ldb)) return -1;
  sA[0] = 1;
  sBpos[0] = 1;
  for (i = 1; i < rank; ++i) {
    sA[i] = sA[i - 1] * (lda ? lda[i - 1] : size[i - 1]);
    sBpos[i] = sBpos[i - 1] * (ldb ? ldb[i - 1] : size[perm[i - 1]]);
  }
  for (j = 0; j < rank; ++j) sB[perm[j]] = sBpos[j];
  int64_t outer = 1;
  for (i = 0; i < rank; ++i) {
    if (size[i] == 0) return 0;
    if (i > 0) outer *= size[i];
  }
  const int ea = esize(type_a), eb = esize(type_b);
  const char* a = (const char*)A;
  char* b = (char*)B;
  const int64_t n0 = size[0];
  int64_t o;
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
  for (o = 0; o < outer; ++o) {
    int64_t rem = o, oa = 0, ob = 0, k;
    int d;
    for (d = 1; d < rank; ++d) {
      const int64_t c = rem % size[d];
      rem /= size[d];
      oa += c * sA[d];
      ob += c * sB[d];
    }
    for (k = 0; k < n0; ++k)
      update(type_a, type_b, beta_nonzero, a + (oa + k) * ea, b + (ob + k * sB[0]) * eb, alpha, beta);
  }
  return 0;
}

#ifdef __cplusplus
}
#endif
