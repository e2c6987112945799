// cc_nufft.cuh — the non-uniform FFT path of the evaluation, for many particles and many modes.
//
// It plays the part of the reference's FINUFFT backend (potential/CollectiveCoordinatePotential.h:119-1250: a type-1
// transform for rho at the constraint modes, type-2 transforms for the forces), built here on the "exponential of
// semicircle" kernel of Barnett, Magland & af Klinteberg (SIAM J. Sci. Comput. 41(5), 2019):
//   phi(t) = exp(beta (sqrt(1 - (2t/w)^2) - 1)),  |t| < w/2 (t in fine-grid units), w = 14, beta = 2.30 w,
// on a fine grid of n_f >= 2 (2K + 1) points per axis (K the largest |n_e| of the k-set). With s the fractional
// coordinates (phase exp(2 pi i n.s)) and x = n_f s:
//   type 1:  f[g] = sum_j prod_e phi(g_e - x_je)   (spread),   F(n) = sum_g f[g] e^{2 pi i n.g / n_f}   (cuFFT),
//            rho(n) = F(n) / prod_e phihat_e(n_e),   phihat(n) = int phi(t) cos(2 pi n t / n_f) dt;
//   type 2:  C[n] = c_n / prod_e phihat_e(n_e),  G[g] = sum_n C[n] e^{2 pi i n.g / n_f}  (cuFFT),
//            v(s_j) = sum_g prod_e phi(g_e - x_je) G[g]  (interpolation),
// with c_n = u_n n_e for the force axis e (u = V conj(rho)) and g_e(j) = Im v(s_j), the integer-index gradient of the
// direct force kernel. Errors are ~1e-13 of sum|c| (measured against direct sums of the same modes).
//
// Determinism: the spread grid accumulates in 64-bit fixed point (scale 2^40) with integer atomics, whose sum does not
// depend on their order; every other sum has a fixed order. Results repeat bitwise.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include "cc_kernels.cuh"

namespace cc {

constexpr int kNufftW = 14;                          // kernel width in fine-grid points
constexpr double kNufftBetaPerW = 2.30;              // beta / w for an upsampling factor of 2
constexpr double kNufftFix = 1099511627776.0;        // 2^40: fixed-point scale of the spread grid
constexpr int kNufftThreads = 128;

struct NufftDev {
	int nf[3];                // fine grid per axis (1 beyond D)
	int K[3];                 // mode half-range per axis
	double beta;
	const double *phihat[3];  // per axis, 2K+1 values for n = -K..K
	int U;                    // unique modes
	const int32_t *umodes;    // U x D
	const double *uV;         // U summed weights
	unsigned long long *gi;   // spread grid (fixed point), nf0 * nf1 * nf2
	double *gr;               // the same as doubles
	const double2 *spec;      // D2Z output: nf0 x nf1 x (nf2/2 + 1) along the last used axis
	double2 *coef;            // D type-2 grids, nf0 * nf1 * nf2 each
	double2 *rho_u, *u_u;     // per unique mode
	double *epart;            // per block of the rho kernel
	const int *skip;
};

__device__ __forceinline__ double es_kernel(double t, double beta)
{
	const double z = 1.0 - (2.0 * t / kNufftW) * (2.0 * t / kNufftW);
	return z > 0.0 ? exp(beta * (sqrt(z) - 1.0)) : 0.0;
}

// kernel weights of one axis for a particle at fine-grid coordinate x: points g0 .. g0 + W - 1
__device__ __forceinline__ int es_weights(double x, double beta, double *k)
{
	const int g0 = (int)ceil(x - 0.5 * kNufftW);
#pragma unroll
	for (int t = 0; t < kNufftW; t++)
		k[t] = es_kernel((double)(g0 + t) - x, beta);
	return g0;
}

__device__ __forceinline__ int wrap_index(int g, int n)
{
	g %= n;
	return g < 0 ? g + n : g;
}

constexpr int kNufftLanes = 16;                    // lanes per particle (kNufftW of them active)
constexpr int kNufftPerBlock = kNufftThreads / kNufftLanes;   // particles per block (two per warp)

// The kernel weights of particle j along every axis into shared memory (lane t < W computes entry t of each axis);
// returns false for a lane without a particle. The 16 lanes of a particle are in one warp.
template <int D>
__device__ __forceinline__ bool nufft_weights(const NufftDev &a, const double *frac, int N, int j, int t,
                                              double (*sk)[kNufftW], int *sg0)
{
	const bool valid = j < N;
	if (valid) {
#pragma unroll
		for (int e = 0; e < D; e++) {
			const double x = frac[(size_t)j * D + e] * a.nf[e];
			const int g0 = (int)ceil(x - 0.5 * kNufftW);
			if (t < kNufftW)
				sk[e][t] = es_kernel((double)(g0 + t) - x, a.beta);
			if (t == 0)
				sg0[e] = g0;
		}
	}
	__syncwarp();
	return valid;
}

// Type-1 spread: 16 lanes per particle; lane t0 adds the particle's weights of first-axis point g0 + t0 to the grid
// in fixed point (integer atomics: the sum does not depend on their order).
template <int D> __global__ void __launch_bounds__(kNufftThreads) nufft_spread_kernel(NufftDev a, const double *frac, int N)
{
	__shared__ double sk[kNufftPerBlock][3][kNufftW];
	__shared__ int sg0[kNufftPerBlock][3];
	if (a.skip && *a.skip)
		return;
	const int p = threadIdx.x / kNufftLanes, t0 = threadIdx.x % kNufftLanes;
	const int j = blockIdx.x * kNufftPerBlock + p;
	if (!nufft_weights<D>(a, frac, N, j, t0, sk[p], sg0[p]) || t0 >= kNufftW)
		return;
	const int i0 = wrap_index(sg0[p][0] + t0, a.nf[0]);
	const double w0 = sk[p][0][t0];
	if constexpr (D == 1) {
		atomicAdd(a.gi + i0, (unsigned long long)llrint(w0 * kNufftFix));
	} else {
		for (int t1 = 0; t1 < kNufftW; t1++) {
			const int i1 = wrap_index(sg0[p][1] + t1, a.nf[1]);
			const double w01 = w0 * sk[p][1][t1];
			if constexpr (D == 2) {
				atomicAdd(a.gi + (size_t)i0 * a.nf[1] + i1, (unsigned long long)llrint(w01 * kNufftFix));
			} else {
				const size_t base = ((size_t)i0 * a.nf[1] + i1) * a.nf[2];
				for (int t2 = 0; t2 < kNufftW; t2++) {
					const int i2 = wrap_index(sg0[p][2] + t2, a.nf[2]);
					atomicAdd(a.gi + base + i2, (unsigned long long)llrint(w01 * sk[p][2][t2] * kNufftFix));
				}
			}
		}
	}
}

static __global__ void nufft_fix_to_double_kernel(NufftDev a, int64_t n)
{
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (a.skip && *a.skip)
		return;
	if (i < n)
		a.gr[i] = (double)a.gi[i] * (1.0 / kNufftFix);
}

__device__ __forceinline__ double phihat_of(const NufftDev &a, int e, int n) { return a.phihat[e][n + a.K[e]]; }

// rho at the unique modes (F_+(n) = conj(F_-(n)) from the D2Z half spectrum, deconvolved), u = V conj(rho), and
// the energy terms summed per block in mode order.
template <int D> __global__ void __launch_bounds__(256) nufft_rho_kernel(NufftDev a, double rho_offset)
{
	__shared__ double sh[8];
	const int u = blockIdx.x * 256 + threadIdx.x;
	if (a.skip && *a.skip)
		return;
	double e = 0.0;
	if (u < a.U) {
		int n[3] = {0, 0, 0};
		double ph = 1.0;
#pragma unroll
		for (int c = 0; c < D; c++) {
			n[c] = a.umodes[(size_t)u * D + c];
			ph *= phihat_of(a, c, n[c]);
		}
		// F_-(m) with m = n, or conj(F_-(-n)) when n's last index lies in the omitted half
		const int L = D - 1, half = a.nf[L] / 2 + 1;
		int m[3];
		bool flip = wrap_index(n[L], a.nf[L]) >= half;
#pragma unroll
		for (int c = 0; c < D; c++)
			m[c] = wrap_index(flip ? -n[c] : n[c], a.nf[c]);
		size_t idx = 0;
#pragma unroll
		for (int c = 0; c < D; c++)
			idx = idx * (c == L ? half : a.nf[c]) + m[c];
		double2 F = a.spec[idx];
		if (flip)
			F.y = -F.y;   // F_-(n) = conj(F_-(-n)) for a real grid
		double2 rho = make_double2(F.x / ph, -F.y / ph);   // rho = F_+(n) / phihat = conj(F_-(n)) / phihat
		rho.x += rho_offset;
		a.rho_u[u] = rho;
		const double v = a.uV[u];
		a.u_u[u] = make_double2(v * rho.x, -v * rho.y);
		e = v * (rho.x * rho.x + rho.y * rho.y);
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		e += __shfl_down_sync(0xffffffffu, e, o);
	if ((threadIdx.x & 31) == 0)
		sh[threadIdx.x >> 5] = e;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < 8; w++)
			t += sh[w];
		a.epart[blockIdx.x] = t;
	}
}

static __global__ void nufft_energy_kernel(NufftDev a, int nblocks, double inv_vol, double shift, double *E_out)
{
	if (a.skip && *a.skip)
		return;
	double e = 0.0;
	for (int b = threadIdx.x; b < nblocks; b += 32)
		e += a.epart[b];
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		e += __shfl_down_sync(0xffffffffu, e, o);
	if (threadIdx.x == 0)
		*E_out = e * inv_vol + shift;
}

// rho in input-mode order from the unique modes
static __global__ void nufft_gather_rho_kernel(const double2 *rho_u, const int *mode_u, int M, double2 *rho_mode)
{
	const int m = blockIdx.x * blockDim.x + threadIdx.x;
	if (m < M)
		rho_mode[m] = rho_u[mode_u[m]];
}

// type-2 coefficients: C_e[n] = u_n n_e / phihat(n) on each axis' grid (the grids were zeroed)
template <int D> __global__ void __launch_bounds__(256) nufft_coef_kernel(NufftDev a, int64_t ngrid)
{
	const int u = blockIdx.x * 256 + threadIdx.x;
	if (a.skip && *a.skip)
		return;
	if (u >= a.U)
		return;
	int n[3] = {0, 0, 0};
	double ph = 1.0;
	size_t idx = 0;
#pragma unroll
	for (int c = 0; c < D; c++) {
		n[c] = a.umodes[(size_t)u * D + c];
		ph *= phihat_of(a, c, n[c]);
		idx = idx * a.nf[c] + wrap_index(n[c], a.nf[c]);
	}
	const double2 uu = a.u_u[u];
#pragma unroll
	for (int c = 0; c < D; c++) {
		const double s = (double)n[c] / ph;
		a.coef[(size_t)c * ngrid + idx] = make_double2(uu.x * s, uu.y * s);
	}
}

struct NufftOut {
	double recip[9];          // reciprocal basis, row e = b_e (Cartesian)
	double fscale;            // 2 / Volume
	double *F_out;            // N x D Cartesian forces, or nullptr
	double *gfrac_out;        // N x D dPhi/ds, or nullptr
};

// type-2 interpolation: 16 lanes per particle; lane t0 sums the first-axis point g0 + t0, the lanes' sums are added
// in a fixed butterfly; g_e = Im(sum_g phi G_e[g]) and the forces as the direct force kernel
template <int D>
__global__ void __launch_bounds__(kNufftThreads) nufft_interp_kernel(NufftDev a, const double *frac, int N,
                                                                     int64_t ngrid, NufftOut o)
{
	__shared__ double sk[kNufftPerBlock][3][kNufftW];
	__shared__ int sg0[kNufftPerBlock][3];
	if (a.skip && *a.skip)
		return;
	const int p = threadIdx.x / kNufftLanes, t0 = threadIdx.x % kNufftLanes;
	const int j = blockIdx.x * kNufftPerBlock + p;
	const bool valid = nufft_weights<D>(a, frac, N, j, t0, sk[p], sg0[p]);
	double acc[D];
#pragma unroll
	for (int e = 0; e < D; e++)
		acc[e] = 0.0;
	if (valid && t0 < kNufftW) {
		const int i0 = wrap_index(sg0[p][0] + t0, a.nf[0]);
		const double w0 = sk[p][0][t0];
		if constexpr (D == 1) {
			acc[0] = w0 * a.coef[i0].y;
		} else {
			for (int t1 = 0; t1 < kNufftW; t1++) {
				const int i1 = wrap_index(sg0[p][1] + t1, a.nf[1]);
				const double w01 = w0 * sk[p][1][t1];
				if constexpr (D == 2) {
					const size_t idx = (size_t)i0 * a.nf[1] + i1;
#pragma unroll
					for (int e = 0; e < D; e++)
						acc[e] = fma(w01, a.coef[(size_t)e * ngrid + idx].y, acc[e]);
				} else {
					const size_t base = ((size_t)i0 * a.nf[1] + i1) * a.nf[2];
					for (int t2 = 0; t2 < kNufftW; t2++) {
						const size_t idx = base + wrap_index(sg0[p][2] + t2, a.nf[2]);
						const double w = w01 * sk[p][2][t2];
#pragma unroll
						for (int e = 0; e < D; e++)
							acc[e] = fma(w, a.coef[(size_t)e * ngrid + idx].y, acc[e]);
					}
				}
			}
		}
	}
#pragma unroll
	for (int off = kNufftLanes / 2; off > 0; off >>= 1)
#pragma unroll
		for (int e = 0; e < D; e++)
			acc[e] += __shfl_xor_sync(0xffffffffu, acc[e], off, kNufftLanes);
	if (valid && t0 == 0)
		write_force_out<D>(o.F_out, o.gfrac_out, o.recip, o.fscale, j, acc);
}

}  // namespace cc
