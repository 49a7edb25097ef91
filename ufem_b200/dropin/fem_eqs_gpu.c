/*
 * fem_eqs_gpu.c -- link-time drop-in of uFEM's linear solver entry points.
 *
 * Defines femEqsCGwJ, femEqsCGwSSOR and femEqsBiCCSwJ with the exact
 * signatures of the reference (fem/fem_math.h:150-152), so the reference's
 * own fem executable or libfem.so links them in place of fem/fem_eqs.c's
 * CPU versions and every caller -- femSolve (fem/fem_sol.c:1722-1730), the
 * Monte Carlo solver (fem/fem_mont.c:498) -- solves on the GPU through
 * libufem_gpu.so, unchanged.  Compile it against the reference's headers:
 *
 *   gcc -c -I<ufem>/fem -I<this repo>/include fem_eqs_gpu.c
 *
 * and link it before the reference objects, with fem_eqs.o's three solver
 * symbols made weak (objcopy --weaken-symbol) or removed, plus
 * -L<repo>/ufem_b200/lib -lufem_gpu.  oracle/Makefile.ref does exactly that
 * for the parity test of the relinked binary.
 *
 * Semantics of the reference kept: a and b/x sizes checked as in
 * fem/fem_eqs.c:103 (AF_ERR_SIZ); x is the in/out initial guess; the
 * stopping rule |r| <= eps (|A| |x| + |b|) with |A| the max row 2-norm;
 * AF_ERR when maxIt runs out, AF_ERR_ZER for a zero diagonal member
 * (femEqsBiCCSwJ returns AF_OK as the reference does).  The matrix must be
 * the reference's row-slot sparse form (MAT_SPAR), the vectors full
 * (VEC_FULL); anything else returns AF_ERR_TYP, as there is no CPU fallback.
 */
#include "fem_math.h"
#include "ufem_gpu.h"

typedef int (*ufem_eqs_fn)(long, const long *, const long *, const long *, const double *, const double *,
                           double *, double, long);

static int gpu_eqs(ufem_eqs_fn fn, tMatrix *a, tVector *b, tVector *x, double eps, long maxIt)
{
  if ((a->cols != x->rows) || (x->rows != b->rows)) return AF_ERR_SIZ; /* fem/fem_eqs.c:103 */
  if (a->type != MAT_SPAR || b->type != VEC_FULL || x->type != VEC_FULL) return AF_ERR_TYP;
  return fn(a->rows, a->frompos, a->defpos, a->pos, a->data, b->data, x->data, eps, maxIt);
}

int femEqsCGwJ(tMatrix *a, tVector *b, tVector *x, double eps, long maxIt)
{
  return gpu_eqs(ufem_eqs_cgwj, a, b, x, eps, maxIt);
}

int femEqsCGwSSOR(tMatrix *a, tVector *b, tVector *x, double eps, long maxIt)
{
  return gpu_eqs(ufem_eqs_cgwssor, a, b, x, eps, maxIt);
}

int femEqsBiCCSwJ(tMatrix *a, tVector *b, tVector *x, double eps, long maxIt)
{
  return gpu_eqs(ufem_eqs_bicgs, a, b, x, eps, maxIt);
}
