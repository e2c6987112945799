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
//   type 2:  C[n] = c_n / prod_e phihat_e(n_e),  G[g] = Im sum_n C[n] e^{2 pi i n.g / n_f}  (cuFFT),
//            v(s_j) = sum_g prod_e phi(g_e - x_je) G[g]  (interpolation),
// with c_n = u_n n_e for the force axis e (u = V conj(rho)) and g_e(j) = v(s_j), the integer-index gradient of the
// direct force kernel. Im sum_n C[n] e^{i theta_n} = sum_n H[n] e^{i theta_n} with the Hermitian
// H[n] = (A[n] + conj(A[-n])) / 2, A = -i C, so G is one complex-to-real transform of H's half spectrum.
// Errors are ~1e-13 of sum|c| (measured against direct sums of the same modes).
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
	double2 *coef;            // D type-2 half spectra H (Z2D input), the D2Z layout each
	double *gim;              // D type-2 real grids G (Z2D output), nf0 * nf1 * nf2 each
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

// the next grid index along an axis of n points, wrapping at n (i in [0, n))
__device__ __forceinline__ int wrap_next(int i, int n) { return i + 1 == n ? 0 : i + 1; }

constexpr int kNufftLanes = 16;                    // lanes per particle (kNufftW of them active): lane t takes the
                                                   // grid points of offset t along the last (contiguous) axis
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

// Type-1 spread: 16 lanes per particle; lane t adds the particle's weights of last-axis point g_last + t, row by row
// of the other axes (a particle's 14 lanes hit 14 consecutive grid words), in fixed point (integer atomics: the sum
// does not depend on their order).
template <int D> __global__ void __launch_bounds__(kNufftThreads) nufft_spread_kernel(NufftDev a, const double *frac, int N)
{
	__shared__ double sk[kNufftPerBlock][3][kNufftW];
	__shared__ int sg0[kNufftPerBlock][3];
	if (a.skip && *a.skip)
		return;
	const int p = threadIdx.x / kNufftLanes, t = threadIdx.x % kNufftLanes;
	const int j = blockIdx.x * kNufftPerBlock + p;
	if (!nufft_weights<D>(a, frac, N, j, t, sk[p], sg0[p]) || t >= kNufftW)
		return;
	constexpr int L = D - 1;
	const int il = wrap_index(sg0[p][L] + t, a.nf[L]);
	const double wl = sk[p][L][t];
	if constexpr (D == 1) {
		atomicAdd(a.gi + il, (unsigned long long)llrint(wl * kNufftFix));
	} else {
		int i0 = wrap_index(sg0[p][0], a.nf[0]);
#pragma unroll 2
		for (int t0 = 0; t0 < kNufftW; t0++, i0 = wrap_next(i0, a.nf[0])) {
			const double w0 = sk[p][0][t0];
			if constexpr (D == 2) {
				atomicAdd(a.gi + (size_t)i0 * a.nf[1] + il, (unsigned long long)llrint(w0 * wl * kNufftFix));
			} else {
				int i1 = wrap_index(sg0[p][1], a.nf[1]);
#pragma unroll 7
				for (int t1 = 0; t1 < kNufftW; t1++, i1 = wrap_next(i1, a.nf[1])) {
					const double w01 = w0 * sk[p][1][t1];
					atomicAdd(a.gi + ((size_t)i0 * a.nf[1] + i1) * a.nf[2] + il,
					          (unsigned long long)llrint(w01 * wl * kNufftFix));
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

// type-2 coefficients: with C_e[n] = u_n n_e / phihat(n) and A = -i C_e, the half spectrum of each axis' Hermitian
// H[m] = (A[m] + conj(A[-m])) / 2 (the spectra were zeroed). Mode n adds A/2 at +n and conj(A)/2 at -n where these lie
// in the stored half (last index 0 .. nf/2). An entry m receives at most two terms (from the modes m and -m, the
// modes being unique), and a sum of two terms onto zero does not depend on their order: the result repeats bitwise.
template <int D> __global__ void __launch_bounds__(256) nufft_coef_kernel(NufftDev a, int64_t nspec)
{
	const int u = blockIdx.x * 256 + threadIdx.x;
	if (a.skip && *a.skip)
		return;
	if (u >= a.U)
		return;
	constexpr int L = D - 1;
	const int half = a.nf[L] / 2 + 1;
	int n[3] = {0, 0, 0};
	double ph = 1.0;
	size_t ip = 0, im = 0;
	bool hp = true, hm = true;
#pragma unroll
	for (int c = 0; c < D; c++) {
		n[c] = a.umodes[(size_t)u * D + c];
		ph *= phihat_of(a, c, n[c]);
		const int mp = wrap_index(n[c], a.nf[c]), mm = wrap_index(-n[c], a.nf[c]);
		if (c == L) {
			hp = mp < half;
			hm = mm < half;
		}
		ip = ip * (c == L ? half : a.nf[c]) + mp;
		im = im * (c == L ? half : a.nf[c]) + mm;
	}
	const double2 uu = a.u_u[u];
#pragma unroll
	for (int c = 0; c < D; c++) {
		const double s = (double)n[c] / ph;
		const double cx = uu.x * s, cy = uu.y * s;   // C = cx + i cy, A = cy - i cx
		double2 *H = a.coef + (size_t)c * nspec;
		if (hp) {
			atomicAdd(&H[ip].x, 0.5 * cy);
			atomicAdd(&H[ip].y, -0.5 * cx);
		}
		if (hm) {
			atomicAdd(&H[im].x, 0.5 * cy);
			atomicAdd(&H[im].y, 0.5 * cx);
		}
	}
}

struct NufftOut {
	double recip[9];          // reciprocal basis, row e = b_e (Cartesian)
	double fscale;            // 2 / Volume
	double *F_out;            // N x D Cartesian forces, or nullptr
	double *gfrac_out;        // N x D dPhi/ds, or nullptr
};

// type-2 interpolation: 16 lanes per particle; lane t sums the last-axis point g_last + t over the rows of the other
// axes (a particle's 14 lanes read 14 consecutive grid words), the lanes' sums are added in a fixed butterfly;
// g_e = sum_g phi G_e[g] and the forces as the direct force kernel
template <int D>
__global__ void __launch_bounds__(kNufftThreads) nufft_interp_kernel(NufftDev a, const double *frac, int N,
                                                                     int64_t ngrid, NufftOut o)
{
	__shared__ double sk[kNufftPerBlock][3][kNufftW];
	__shared__ int sg0[kNufftPerBlock][3];
	if (a.skip && *a.skip)
		return;
	const int p = threadIdx.x / kNufftLanes, t = threadIdx.x % kNufftLanes;
	const int j = blockIdx.x * kNufftPerBlock + p;
	const bool valid = nufft_weights<D>(a, frac, N, j, t, sk[p], sg0[p]);
	double acc[D];
#pragma unroll
	for (int e = 0; e < D; e++)
		acc[e] = 0.0;
	if (valid && t < kNufftW) {
		constexpr int L = D - 1;
		const int il = wrap_index(sg0[p][L] + t, a.nf[L]);
		const double wl = sk[p][L][t];
		if constexpr (D == 1) {
			acc[0] = wl * a.gim[il];
		} else if constexpr (D == 2) {
			// all rows' loads issued before the sums (the row indices wrap incrementally)
			int i0 = wrap_index(sg0[p][0], a.nf[0]);
			double v[kNufftW][D];
#pragma unroll
			for (int t0 = 0; t0 < kNufftW; t0++, i0 = wrap_next(i0, a.nf[0])) {
				const size_t idx = (size_t)i0 * a.nf[1] + il;
#pragma unroll
				for (int e = 0; e < D; e++)
					v[t0][e] = __ldg(a.gim + (size_t)e * ngrid + idx);
			}
#pragma unroll
			for (int t0 = 0; t0 < kNufftW; t0++) {
				const double w = sk[p][0][t0] * wl;
#pragma unroll
				for (int e = 0; e < D; e++)
					acc[e] = fma(w, v[t0][e], acc[e]);
			}
		} else {
			int i0 = wrap_index(sg0[p][0], a.nf[0]);
			const int i1s = wrap_index(sg0[p][1], a.nf[1]);
			for (int t0 = 0; t0 < kNufftW; t0++, i0 = wrap_next(i0, a.nf[0])) {
				const double w0 = sk[p][0][t0];
				int i1 = i1s;
				double v[kNufftW][D];
#pragma unroll
				for (int t1 = 0; t1 < kNufftW; t1++, i1 = wrap_next(i1, a.nf[1])) {
					const size_t idx = ((size_t)i0 * a.nf[1] + i1) * a.nf[2] + il;
#pragma unroll
					for (int e = 0; e < D; e++)
						v[t1][e] = __ldg(a.gim + (size_t)e * ngrid + idx);
				}
#pragma unroll
				for (int t1 = 0; t1 < kNufftW; t1++) {
					const double w = w0 * sk[p][1][t1] * wl;
#pragma unroll
					for (int e = 0; e < D; e++)
						acc[e] = fma(w, v[t1][e], acc[e]);
				}
			}
		}
	}
#pragma unroll
	for (int off = kNufftLanes / 2; off > 0; off >>= 1)
#pragma unroll
		for (int e = 0; e < D; e++)
			acc[e] += __shfl_xor_sync(0xffffffffu, acc[e], off, kNufftLanes);
	if (valid && t == 0)
		write_force_out<D>(o.F_out, o.gfrac_out, o.recip, o.fscale, j, acc);
}

}  // namespace cc
