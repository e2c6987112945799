/* ORACLE — test infrastructure, not product code.
 *
 * Plain-C restatement of the reference's collective-coordinate direct sums, used only as a checker by the tests,
 * the smoke check and the CPU-baseline leg of bench.py. It never runs on the product path.
 *
 * Each function follows the reference's arithmetic order so that, built with -ffp-contract=off, it reproduces the
 * reference's FP64 results to rounding level (it is pinned against the reference itself, compiled from its own
 * sources into oracle/_ref, and against the committed golden vectors made from it):
 *   cco_cartesian  core/PeriodicCellList.h:517-538 (relative coordinate wrapped by floor twice) and :88-98
 *                  (Cartesian = sum_i s_i a_i, accumulated in basis order);
 *   cco_rho        potential/CollectiveCoordinatePotential.h:1255-1286 (GetRho_Direct: per k, particles in order,
 *                  cos and sin of the d-term dot product k.r);
 *   cco_energy     :1351-1372 (sum_k V_k (Re^2 + Im^2), then / Volume + Shift);
 *   cco_forces     :1377-1394 (Force: F_i -= 2 V_k (Im cos(k.r) - Re sin(k.r)) k, in k order, then * 1/Volume);
 *   cco_sk         pairstat/StructureFactor.cpp:56-65 (|sum_j exp(i k.r_j)|^2 / N).
 * The volume is |det| of the basis (core/GeometryVector.cpp:63-77 computes it through an LU factorisation).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

static double dot(int d, const double *a, const double *b)
{
	double r = 0;
	for (int i = 0; i < d; i++)
		r += a[i] * b[i];
	return r;
}

double cco_volume(int d, const double *basis)
{
	if (d == 1)
		return fabs(basis[0]);
	if (d == 2)
		return fabs(basis[0] * basis[3] - basis[1] * basis[2]);
	if (d == 3) {
		const double *a = basis, *b = basis + 3, *c = basis + 6;
		return fabs(a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
		            a[2] * (b[0] * c[1] - b[1] * c[0]));
	}
	return NAN;
}

/* out (N x d): Cartesian coordinates of the fractional positions frac (N x d), wrapped into [0,1) first. */
void cco_cartesian(int d, const double *basis, long N, const double *frac, double *out)
{
	for (long j = 0; j < N; j++) {
		double s[4];
		for (int i = 0; i < d; i++) {
			s[i] = frac[j * d + i] - floor(frac[j * d + i]);
			s[i] -= floor(s[i]);
		}
		for (int c = 0; c < d; c++)
			out[j * d + c] = 0.0;
		for (int i = 0; i < d; i++)
			for (int c = 0; c < d; c++)
				out[j * d + c] += basis[i * d + c] * s[i];
	}
}

/* rho over M Cartesian k (M x d) for N Cartesian positions r (N x d). */
void cco_rho(int d, long N, const double *r, long M, const double *k, double *re, double *im)
{
#pragma omp parallel for schedule(static)
	for (long q = 0; q < M; q++) {
		double tr = 0, ti = 0;
		for (long j = 0; j < N; j++) {
			tr += cos(dot(d, k + q * d, r + j * d));
			ti += sin(dot(d, k + q * d, r + j * d));
		}
		re[q] = tr;
		im[q] = ti;
	}
}

double cco_energy(long M, const double *V, const double *re, const double *im, double volume, double shift)
{
	double e = 0;
	for (long q = 0; q < M; q++)
		e += V[q] * (re[q] * re[q] + im[q] * im[q]);
	return e / volume + shift;
}

/* Cartesian forces (N x d) given rho. */
void cco_forces(int d, long N, const double *r, long M, const double *k, const double *V, const double *re,
                const double *im, double volume, double *F)
{
#pragma omp parallel for schedule(static)
	for (long j = 0; j < N; j++) {
		double f[4] = {0, 0, 0, 0};
		for (long q = 0; q < M; q++) {
			const double *kq = k + q * d;
			double s = 2.0 * V[q] * (im[q] * cos(dot(d, kq, r + j * d)) - re[q] * sin(dot(d, kq, r + j * d)));
			for (int c = 0; c < d; c++)
				f[c] -= s * kq[c];
		}
		for (int c = 0; c < d; c++)
			F[j * d + c] = f[c] * (1.0 / volume);
	}
}

/* One full evaluation from fractional positions: returns the energy; F, re, im may be NULL. */
double cco_eval(int d, const double *basis, long N, const double *frac, long M, const double *k, const double *V,
                double shift, double *F, double *re, double *im)
{
	double *r = (double *)malloc(sizeof(double) * (size_t)(N * d + 1));
	double *wr = re ? re : (double *)malloc(sizeof(double) * (size_t)(M + 1));
	double *wi = im ? im : (double *)malloc(sizeof(double) * (size_t)(M + 1));
	cco_cartesian(d, basis, N, frac, r);
	cco_rho(d, N, r, M, k, wr, wi);
	double vol = cco_volume(d, basis);
	double e = cco_energy(M, V, wr, wi, vol, shift);
	if (F)
		cco_forces(d, N, r, M, k, V, wr, wi, vol, F);
	free(r);
	if (!re)
		free(wr);
	if (!im)
		free(wi);
	return e;
}

/* S(k) for K Cartesian wavevectors from fractional positions. */
void cco_sk(int d, const double *basis, long N, const double *frac, long K, const double *k, double *S)
{
	double *r = (double *)malloc(sizeof(double) * (size_t)(N * d + 1));
	cco_cartesian(d, basis, N, frac, r);
#pragma omp parallel for schedule(guided)
	for (long q = 0; q < K; q++) {
		double tr = 0, ti = 0;
		for (long j = 0; j < N; j++) {
			double p = dot(d, k + q * d, r + j * d);
			tr += cos(p);
			ti += sin(p);
		}
		S[q] = (tr * tr + ti * ti) / (double)N;
	}
	free(r);
}
