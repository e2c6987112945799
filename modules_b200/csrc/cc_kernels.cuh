// cc_kernels.cuh — sm_100a kernels of the collective-coordinate (CC) potential.
//
// Work decomposition. The constraint modes n (integer k-lattice indices) are grouped on the host into SEGMENTS: up
// to L modes that share every index but the last and whose last index runs start, start+1, ..., start+len-1 (a piece
// of a lattice line). For one particle with fractional coordinates s, the phases of a segment are
//     z_r = exp(2 pi i n_r.s) = z_0 * w^r,   z_0 = exp(2 pi i (prefix.s' + start s_last)),  w = exp(2 pi i s_last),
// so one seed (an exactly reduced sincospi) gives L phases through complex multiplications, which are FMA work.
// A segment owns L consecutive SLOTS; slot values are the per-segment rho partials, and every input mode maps to
// one slot (repeated modes share it). Empty slots (r >= len, padding segments) carry weight 0.
//
// rho pass (cc_rho_kernel): one lane per segment, a block = 32 segments (its GROUP) x WARPS warps that stride over
// the block's particle range; particles are staged in shared memory and read as warp-wide broadcasts. The warps'
// accumulators are summed in a fixed order, written as the block's partial, and the last block of each group (an
// atomic ticket, no waiting) sums the partials of all particle splits in split order. The last group overall forms
// the energy sum over modes in mode order. Every sum has a fixed order, so results repeat bitwise.
//
// force pass (cc_force_kernel): one lane per particle, a block = 32 particles x WARPS warps that stride over the
// block's segment range; segment descriptors and weights u = V conj(rho) are staged in shared memory and read as
// broadcasts. Per segment the lane accumulates S0 = sum_r t_r and S1 = sum_r r t_r with t_r = Im(u_r z_r); the
// integer-index gradient is g += S0 * (prefix, start) + (0.., S1). Cartesian force F = (2/V) sum_e g_e b_e; the
// gradient in fractional coordinates is dPhi/ds_e = -(2/V) 2 pi g_e.
//
// Precision. FP64 path: phases from an exact argument reduction of n.s modulo 1 (two-product with FMA, integer parts
// removed by rint), FP64 sincospi seeds, FP64 recurrences and sums. Mixed path: the same FP64 reduction, then FP32
// sincospi seeds and FP32 recurrences; per-lane FP32 sums are flushed into FP64 accumulators every SUB particles
// (rho) or every segment (force), and all cross-lane sums are FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

#include "cc_plan.h"

namespace cc {


// ---------------------------------------------------------------------------------------------------------------
// exact fractional phase: t = (sum_e n_e s_e) mod 1, in [-1/2, 1/2]
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void acc_phase(int n, double s, double &hi, double &lo)
{
	const double nd = (double)n;
	const double p = __dmul_rn(nd, s);
	lo = __dadd_rn(lo, __fma_rn(nd, s, -p));          // exact rounding error of the product
	hi = __dadd_rn(hi, __dsub_rn(p, rint(p)));        // exact: fractional part of the rounded product
}

template <int D>
__device__ __forceinline__ double seg_phase(const Seg &g, const double *s)
{
	double hi = 0.0, lo = 0.0;
	if (D >= 2)
		acc_phase(g.p0, s[0], hi, lo);
	if (D >= 3)
		acc_phase(g.p1, s[1], hi, lo);
	acc_phase(g.start, s[D - 1], hi, lo);
	const double t = __dadd_rn(hi, lo);
	return __dsub_rn(t, rint(t));
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
	return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
	return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// exp(2 pi i t) for t in [-1/2, 1/2] (or [0,1)): (cos, sin)
__device__ __forceinline__ double2 expi2pi(double t)
{
	double s, c;
	sincospi(2.0 * t, &s, &c);
	return make_double2(c, s);
}
__device__ __forceinline__ float2 expi2pif(double t)
{
	float s, c;
	sincospif(2.0f * (float)t, &s, &c);
	return make_float2(c, s);
}

template <typename T> struct Cx;
template <> struct Cx<double> {
	typedef double2 type;
	static __device__ __forceinline__ double2 expi(double t) { return expi2pi(t); }
	static __device__ __forceinline__ double2 mul(double2 a, double2 b) { return cmul(a, b); }
	static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
};
template <> struct Cx<float> {
	typedef float2 type;
	static __device__ __forceinline__ float2 expi(double t) { return expi2pif(t); }
	static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return cmulf(a, b); }
	static __device__ __forceinline__ float2 zero() { return make_float2(0.0f, 0.0f); }
};

// ---------------------------------------------------------------------------------------------------------------
// parameters
// ---------------------------------------------------------------------------------------------------------------
struct RhoArgs {
	const double *frac;       // N x D fractional coordinates in [0,1)
	int N;
	int per_split;            // particles per block (blockIdx.y)
	int nsplit;
	const Seg *segs;          // ngroups*32 segments
	int ngroups;
	int nslot;                // ngroups*32*L
	double2 *partial;         // [nsplit][nslot]
	unsigned *counters;       // [ngroups + 1], zero between launches
	double2 *rho_slot;        // [nslot]
	const double *slotV;      // [nslot] summed weight of the modes in the slot
	double2 *u_slot;          // [nslot] u = slotV * conj(rho)
	const int *mode_slot;     // [M]
	const double *modeV;      // [M]
	int M;
	double rho_offset;        // added to Re rho of every slot
	double inv_vol, shift;
	double *E_out;            // energy (device scalar)
	double2 *rho_mode;        // [M] rho in mode order, or nullptr
};

struct ForceArgs {
	const double *frac;       // N x D
	int N;
	const Seg *segs;
	int nseg;                 // ngroups*32
	int segs_per_split;
	int nksplit;
	const double2 *u_slot;    // [nseg*L]
	double *partialG;         // [nksplit][N][D], only for nksplit > 1
	unsigned *counters;       // [ceil(N/32)], zero between launches
	double recip[9];          // reciprocal basis, row e = b_e (Cartesian)
	double fscale;            // 2 / Volume
	double *F_out;            // N x D Cartesian forces, or nullptr
	double *gfrac_out;        // N x D dPhi/ds, or nullptr
};

// ---------------------------------------------------------------------------------------------------------------
// rho pass
// ---------------------------------------------------------------------------------------------------------------
// dynamic shared memory layout of cc_rho_kernel (16-byte aligned pieces)
template <int D, int L, int WARPS, int CHUNK, bool MIXED>
struct RhoSmem {
	static constexpr size_t al(size_t x) { return (x + 15) & ~size_t(15); }
	static constexpr size_t off_s = 0;
	static constexpr size_t off_w = al(sizeof(double) * CHUNK * D);
	static constexpr size_t off_red = al(off_w + (MIXED ? sizeof(float2) : sizeof(double2)) * CHUNK);
	static constexpr size_t bytes = al(off_red + sizeof(double2) * WARPS * 32 * L);
};

// per-particle recurrence step w = exp(2 pi i s_last): computed in FP64 and rounded for the mixed path
template <typename R> __device__ __forceinline__ typename Cx<R>::type step_w(double s);
template <> __device__ __forceinline__ double2 step_w<double>(double s) { return expi2pi(s); }
template <> __device__ __forceinline__ float2 step_w<float>(double s)
{
	const double2 w = expi2pi(s);
	return make_float2((float)w.x, (float)w.y);
}

template <int D, int L, int WARPS, int CHUNK, bool MIXED>
__global__ void __launch_bounds__(WARPS * 32) cc_rho_kernel(RhoArgs a)
{
	typedef typename std::conditional<MIXED, float, double>::type R;
	typedef typename Cx<R>::type C;
	constexpr int SUB = 32;   // mixed: FP32 partial sums are flushed to FP64 after this many particles per lane

	extern __shared__ __align__(16) unsigned char smem[];
	typedef RhoSmem<D, L, WARPS, CHUNK, MIXED> Lay;
	double *sh_s = reinterpret_cast<double *>(smem + Lay::off_s);     // CHUNK*D
	C *sh_w = reinterpret_cast<C *>(smem + Lay::off_w);               // CHUNK
	double2 *sh_red = reinterpret_cast<double2 *>(smem + Lay::off_red); // WARPS*32*L
	__shared__ int sh_last;

	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int group = blockIdx.x, split = blockIdx.y;
	const Seg sg = a.segs[group * 32 + lane];
	const int j0 = split * a.per_split;
	const int j1 = min(a.N, j0 + a.per_split);

	double2 acc[L];
#pragma unroll
	for (int r = 0; r < L; r++)
		acc[r] = make_double2(0.0, 0.0);
	C accf[L];
	int since_flush = 0;
	if (MIXED) {
#pragma unroll
		for (int r = 0; r < L; r++)
			accf[r] = Cx<R>::zero();
	}

	for (int cj = j0; cj < j1; cj += CHUNK) {
		const int cnt = min(CHUNK, j1 - cj);
		__syncthreads();
		for (int i = threadIdx.x; i < cnt; i += WARPS * 32) {
#pragma unroll
			for (int e = 0; e < D; e++)
				sh_s[i * D + e] = a.frac[(size_t)(cj + i) * D + e];
			sh_w[i] = step_w<R>(a.frac[(size_t)(cj + i) * D + D - 1]);
		}
		__syncthreads();
		for (int i = warp; i < cnt; i += WARPS) {
			double s[D];
#pragma unroll
			for (int e = 0; e < D; e++)
				s[e] = sh_s[i * D + e];
			const C w = sh_w[i];
			C z = Cx<R>::expi(seg_phase<D>(sg, s));
			if (MIXED) {
#pragma unroll
				for (int r = 0; r < L; r++) {
					accf[r].x += z.x;
					accf[r].y += z.y;
					z = Cx<R>::mul(z, w);
				}
				if (++since_flush == SUB) {
					since_flush = 0;
#pragma unroll
					for (int r = 0; r < L; r++) {
						acc[r].x += (double)accf[r].x;
						acc[r].y += (double)accf[r].y;
						accf[r] = Cx<R>::zero();
					}
				}
			} else {
#pragma unroll
				for (int r = 0; r < L; r++) {
					acc[r].x += (double)z.x;
					acc[r].y += (double)z.y;
					z = Cx<R>::mul(z, w);
				}
			}
		}
	}
	if (MIXED) {
#pragma unroll
		for (int r = 0; r < L; r++) {
			acc[r].x += (double)accf[r].x;
			acc[r].y += (double)accf[r].y;
		}
	}

	// fixed-order sum over the block's warps
	__syncthreads();
#pragma unroll
	for (int r = 0; r < L; r++)
		sh_red[(warp * 32 + lane) * L + r] = acc[r];
	__syncthreads();
	const size_t gbase = (size_t)group * 32 * L;
	for (int q = threadIdx.x; q < 32 * L; q += WARPS * 32) {
		double2 t = sh_red[q];
		for (int w = 1; w < WARPS; w++) {
			const double2 v = sh_red[w * 32 * L + q];
			t.x += v.x;
			t.y += v.y;
		}
		a.partial[(size_t)split * a.nslot + gbase + q] = t;
	}

	// the last block of this group sums the partials of every split, in split order
	__threadfence();
	__syncthreads();
	if (threadIdx.x == 0)
		sh_last = (atomicAdd(&a.counters[group], 1u) == (unsigned)(a.nsplit - 1));
	__syncthreads();
	if (!sh_last)
		return;
	__threadfence();
	for (int q = threadIdx.x; q < 32 * L; q += WARPS * 32) {
		double2 t = __ldcg(&a.partial[gbase + q]);
		for (int sp = 1; sp < a.nsplit; sp++) {
			const double2 v = __ldcg(&a.partial[(size_t)sp * a.nslot + gbase + q]);
			t.x += v.x;
			t.y += v.y;
		}
		t.x += a.rho_offset;
		a.rho_slot[gbase + q] = t;
		const double v = a.slotV[gbase + q];
		a.u_slot[gbase + q] = make_double2(v * t.x, -v * t.y);
	}
	if (threadIdx.x == 0)
		a.counters[group] = 0u;

	// the last group overall forms the energy in mode order
	__threadfence();
	__syncthreads();
	if (threadIdx.x == 0)
		sh_last = (atomicAdd(&a.counters[a.ngroups], 1u) == (unsigned)(a.ngroups - 1));
	__syncthreads();
	if (!sh_last)
		return;
	__threadfence();
	double e = 0.0;
	for (int m = threadIdx.x; m < a.M; m += WARPS * 32) {
		const double2 rho = __ldcg(&a.rho_slot[a.mode_slot[m]]);
		e += a.modeV[m] * (rho.x * rho.x + rho.y * rho.y);
		if (a.rho_mode)
			a.rho_mode[m] = rho;
	}
	__syncthreads();
	double *sh_e = reinterpret_cast<double *>(sh_red);
	sh_e[threadIdx.x] = e;
	__syncthreads();
	for (int stride = WARPS * 16; stride > 0; stride >>= 1) {
		if (threadIdx.x < stride)
			sh_e[threadIdx.x] += sh_e[threadIdx.x + stride];
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		*a.E_out = sh_e[0] * a.inv_vol + a.shift;
		a.counters[a.ngroups] = 0u;
	}
}

// ---------------------------------------------------------------------------------------------------------------
// force pass
// ---------------------------------------------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void write_force(const ForceArgs &a, int j, const double *g)
{
	if (a.F_out) {
#pragma unroll
		for (int c = 0; c < D; c++) {
			double f = 0.0;
#pragma unroll
			for (int e = 0; e < D; e++)
				f = fma(g[e], a.recip[e * D + c], f);
			a.F_out[(size_t)j * D + c] = a.fscale * f;
		}
	}
	if (a.gfrac_out) {
		const double gs = -a.fscale * 6.283185307179586476925286766559;
#pragma unroll
		for (int e = 0; e < D; e++)
			a.gfrac_out[(size_t)j * D + e] = gs * g[e];
	}
}

template <int D, int L, int WARPS, int SEGCHUNK, bool MIXED>
__global__ void __launch_bounds__(WARPS * 32) cc_force_kernel(ForceArgs a)
{
	typedef typename std::conditional<MIXED, float, double>::type R;
	typedef typename Cx<R>::type C;
	__shared__ Seg sh_seg[SEGCHUNK];
	__shared__ C sh_u[SEGCHUNK * L];
	__shared__ double sh_g[WARPS * 32 * D];
	__shared__ int sh_last;

	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int j = blockIdx.x * 32 + lane;
	const int ks = blockIdx.y;
	const int q0 = ks * a.segs_per_split;
	const int q1 = min(a.nseg, q0 + a.segs_per_split);

	double s[D];
#pragma unroll
	for (int e = 0; e < D; e++)
		s[e] = (j < a.N) ? a.frac[(size_t)j * D + e] : 0.0;
	const C w = step_w<R>(s[D - 1]);

	double g[D];
#pragma unroll
	for (int e = 0; e < D; e++)
		g[e] = 0.0;

	for (int cq = q0; cq < q1; cq += SEGCHUNK) {
		const int cnt = min(SEGCHUNK, q1 - cq);
		__syncthreads();
		for (int i = threadIdx.x; i < cnt; i += WARPS * 32)
			sh_seg[i] = a.segs[cq + i];
		for (int i = threadIdx.x; i < cnt * L; i += WARPS * 32) {
			const double2 u = a.u_slot[(size_t)cq * L + i];
			if (MIXED)
				reinterpret_cast<float2 *>(sh_u)[i] = make_float2((float)u.x, (float)u.y);
			else
				reinterpret_cast<double2 *>(sh_u)[i] = u;
		}
		__syncthreads();
		for (int q = warp; q < cnt; q += WARPS) {
			const Seg sg = sh_seg[q];
			if (sg.len == 0)
				continue;
			C z = Cx<R>::expi(seg_phase<D>(sg, s));
			R S0 = 0, S1 = 0;
#pragma unroll
			for (int r = 0; r < L; r++) {
				const C u = sh_u[q * L + r];
				const R t = u.x * z.y + u.y * z.x;
				S0 += t;
				S1 = fma((R)r, t, S1);
				z = Cx<R>::mul(z, w);
			}
			const double S0d = (double)S0;
			if (D >= 2)
				g[0] = fma(S0d, (double)sg.p0, g[0]);
			if (D >= 3)
				g[1] = fma(S0d, (double)sg.p1, g[1]);
			g[D - 1] = fma(S0d, (double)sg.start, g[D - 1] + (double)S1);
		}
	}

	// fixed-order sum over the block's warps
	__syncthreads();
#pragma unroll
	for (int e = 0; e < D; e++)
		sh_g[(warp * 32 + lane) * D + e] = g[e];
	__syncthreads();
	if (warp != 0)
		return;
	double t[D];
#pragma unroll
	for (int e = 0; e < D; e++) {
		t[e] = sh_g[lane * D + e];
		for (int w2 = 1; w2 < WARPS; w2++)
			t[e] += sh_g[(w2 * 32 + lane) * D + e];
	}
	if (a.nksplit == 1) {
		if (j < a.N)
			write_force<D>(a, j, t);
		return;
	}
	if (j < a.N) {
#pragma unroll
		for (int e = 0; e < D; e++)
			a.partialG[((size_t)ks * a.N + j) * D + e] = t[e];
	}
	__threadfence();
	__syncwarp();
	if (lane == 0)
		sh_last = (atomicAdd(&a.counters[blockIdx.x], 1u) == (unsigned)(a.nksplit - 1));
	__syncwarp();
	if (!sh_last)
		return;
	__threadfence();
	if (j < a.N) {
		double u[D];
#pragma unroll
		for (int e = 0; e < D; e++)
			u[e] = __ldcg(&a.partialG[(size_t)j * D + e]);
		for (int k2 = 1; k2 < a.nksplit; k2++)
#pragma unroll
			for (int e = 0; e < D; e++)
				u[e] += __ldcg(&a.partialG[((size_t)k2 * a.N + j) * D + e]);
		write_force<D>(a, j, u);
	}
	if (lane == 0)
		a.counters[blockIdx.x] = 0u;
}

}  // namespace cc
