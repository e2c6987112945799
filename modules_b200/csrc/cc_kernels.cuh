// cc_kernels.cuh — sm_100a kernels of the collective-coordinate (CC) potential.
//
// Work decomposition. The constraint modes n (integer k-lattice indices) are grouped on the host into SEGMENTS of
// L = 8 modes that share every index but the last and whose last index runs start, start+1, ... (a piece of a lattice
// line). For a particle with fractional coordinates s the phases of a segment are
//     z_r = exp(2 pi i n_r.s) = z_0 w^r,   w = exp(2 pi i s_last),
// so after one seed z_0 every further phase is one step of a recurrence (FMA work: the three-term recurrence in FP64,
// a complex product in the mixed path). Seeds come from per-particle
// PHASE TABLES built in shared memory for the block's particles: T_e(m) = exp(2 pi i m s_e) over the index range the
// block's segments use, either in full or as coarse (stride 8) x fine (0..7) factors; each 8-entry block of a table
// starts from an exactly reduced FP64 sincospi and continues by at most 7 FP64 complex multiplications, so table
// entries are accurate to a few ulp whatever the index. A seed is then 2-3 complex products of table entries.
//
// Exact argument reduction: n.s mod 1 is formed from the rounded product and its exact FMA residual, with the integer
// part removed by rint, so the phase carries ~1e-16 of a turn of error for any |n| (the reference forms k.r in
// Cartesian coordinates, whose rounding grows with |k.r|).
//
// Per evaluation (FP64 or mixed), every kernel 256 threads:
//   cc_rho_kernel    grid (block groups x particle splits), thread-block clusters of up to 8 splits. Warp w owns the
//                    32 segments of one rho group (a lane per segment); all warps walk the block's particles, whose
//                    tables are built per chunk in shared memory. The cluster's blocks add their sums through
//                    distributed shared memory into one partial row of every slot.
//   cc_reduce_kernel sums the partial rows of every slot in row order (8 chunks in parallel, combined in chunk order),
//                    forms rho, u = V conj(rho) and one energy term per block (summed in block order by the force
//                    kernel, or by the reduce kernel's last block, which takes an atomic ticket and never waits).
//   cc_force_kernel  grid (particle groups of 32 x segment splits): 32 particles (lanes) x 8 warps sharing the split's
//                    segments, whose weights u are staged 128 segments at a time. Per segment: S0 = sum_r t_r,
//                    S1 = sum_r r t_r with t_r = Im(u_r z_r); the integer-index gradient is g += S0 (prefix, start)
//                    + (0, S1). In FP64 a warp takes a contiguous run of segments and continues the recurrence along a
//                    lattice line for up to kForceRun segments. Splits are summed in split order by the last block of
//                    each particle group. Cartesian F = (2/V) sum_e g_e b_e; dPhi/ds_e = -(2/V) 2 pi g_e.
//   The kernels are chained by programmatic dependent launch: each is scheduled while its predecessor drains and
//   waits for it (cudaGridDependencySynchronize) before reading its results.
//   cc_mbatch_kernel: the same block bodies for many instances (any dimensions) in ONE persistent launch, items
//   (instance, phase, block) taken from one work queue, the phases of an instance ordered by completion counts.
// Every sum has a fixed order, so results repeat bitwise.
//
// Mixed precision: table entries are FP32 sincospi of the exactly reduced FP64 arguments, continued by FP32 products
// within each 8-entry block; seeds and the three-term recurrence along a segment run in FP32; per-thread rho sums are
// flushed to FP64 every 16 particles, per-segment force sums are added to FP64; all cross-thread sums are FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cooperative_groups.h>
#include <type_traits>

#include "cc_plan.h"

namespace cc {

namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------------------------------------------
// exact fractional phase
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void acc_phase(int n, double s, double &hi, double &lo)
{
	const double nd = (double)n;
	const double p = __dmul_rn(nd, s);
	lo = __dadd_rn(lo, __fma_rn(nd, s, -p));          // exact rounding error of the product
	hi = __dadd_rn(hi, __dsub_rn(p, rint(p)));        // exact: fractional part of the rounded product
}

// (n . s) mod 1 in [-1/2, 1/2] for a segment's first mode
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

// (m s) mod 1 in [-1/2, 1/2]
__device__ __forceinline__ double phase1(int m, double s)
{
	double hi = 0.0, lo = 0.0;
	acc_phase(m, s, hi, lo);
	const double t = __dadd_rn(hi, lo);
	return __dsub_rn(t, rint(t));
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
	return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
	return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// Three-term recurrence along a lattice line: z_{r+1} = c z_r - z_{r-1} with c = 2 cos(theta), for z_r = z_0 w^r and
// w = exp(i theta) (z_{r+1} + z_{r-1} = (w + 1/w) z_r). Two FMAs per step instead of a complex product; the rounding
// error of step r is amplified by at most |sin(r theta) / sin(theta)| <= r, so a line of L slots stays within
// ~L^2/2 ulps.
__device__ __forceinline__ double2 cheb_next(double c, double2 q, double2 p)
{
	return make_double2(fma(c, q.x, -p.x), fma(c, q.y, -p.y));
}

// acc += a + b (a, b: the same slot of two particles) and acc += a, component by component; the FP32 forms are packed
// FP32x2 adds with the scalar adds' rounding, so both forms give the same sums.
__device__ __forceinline__ void acc_add(double2 &acc, double2 a, double2 b)
{
	acc.x += a.x + b.x;
	acc.y += a.y + b.y;
}
__device__ __forceinline__ void acc_add(float2 &acc, float2 a, float2 b) { acc = __fadd2_rn(acc, __fadd2_rn(a, b)); }
__device__ __forceinline__ void acc_add(double2 &acc, double2 a)
{
	acc.x += a.x;
	acc.y += a.y;
}
__device__ __forceinline__ void acc_add(float2 &acc, float2 a) { acc = __fadd2_rn(acc, a); }

// The FP32 recurrence (the mixed path; a segment of L = 8 slots stays within ~L^2/2 = 32 FP32 ulps of its seed's
// phase), both components in one packed FP32x2 fused multiply-add (sm_100) rounded as fmaf, and written without a
// negated addend: y_r = s_r z_r with s_r = -1 for r mod 4 in {2, 3} obeys
// y_r = -c y_{r-1} + y_{r-2} for even r and y_r = c y_{r-1} + y_{r-2} for odd r. Negation is exact and commutes with
// round-to-nearest, so y_r is s_r z_r bit for bit (and so are sums of y_r). cpos = (c, c), cneg = (-c, -c).
__host__ __device__ constexpr bool slot_negated(int r) { return (r & 2) != 0; }
// (called from fully unrolled loops, where r is a constant and the choice is made at compile time)
__device__ __forceinline__ float2 seg_next(int r, float2 cpos, float2 cneg, float2 q, float2 p)
{
	return __ffma2_rn((r & 1) ? cpos : cneg, q, p);
}

// exp(2 pi i t): (cos, sin)
__device__ __forceinline__ double2 expi2pi(double t)
{
	double s, c;
	sincospi(2.0 * t, &s, &c);
	return make_double2(c, s);
}
// exp(2 pi i t) in FP32 for an exactly reduced argument t in [-1/2, 1/2] (rounded once to FP32, ~3e-8 of a turn)
__device__ __forceinline__ float2 expi2pi_f(double t)
{
	float s, c;
	sincospif(2.0f * (float)t, &s, &c);
	return make_float2(c, s);
}

template <typename C> __device__ __forceinline__ C to_c(double2 z);
template <> __device__ __forceinline__ double2 to_c<double2>(double2 z) { return z; }
template <> __device__ __forceinline__ float2 to_c<float2>(double2 z) { return make_float2((float)z.x, (float)z.y); }

// ---------------------------------------------------------------------------------------------------------------
// phase tables
// ---------------------------------------------------------------------------------------------------------------
// Build the tables of `cnt` particles (fractional coordinates frac[(first + i) * D + axis], i < nvalid; rows of the
// remaining particles get the tables of s = 0) into tab. Entry k of particle i lives at tab[i * pstride + k * estride].
// One work item = up to 8 consecutive entries of one run.
template <int D, typename C>
__device__ __forceinline__ void build_tables(const TabSpec &sp, const double *__restrict__ frac, int64_t first,
                                             int cnt, int nvalid, C *tab, int pstride, int estride, int tid,
                                             int nthreads)
{
	const int total = cnt * sp.items;
	for (int t = tid; t < total; t += nthreads) {
		const int i = t / sp.items;
		int k = t - i * sp.items;
		int r = 0;
		int nb = (sp.run[0].count + 7) >> 3;
		while (k >= nb) {
			k -= nb;
			r++;
			nb = (sp.run[r].count + 7) >> 3;
		}
		const TabRun &run = sp.run[r];
		const double s = (i < nvalid) ? frac[(first + i) * D + run.axis] : 0.0;
		const int k0 = k * 8;
		const int k1 = min(run.count, k0 + 8);
		C *dst = tab + (size_t)i * pstride;
		if constexpr (std::is_same<C, float2>::value) {
			// mixed precision: FP32 sincospi of the exactly reduced FP64 argument, FP32 products along the block
			float2 z = expi2pi_f(phase1(run.m0 + run.stride * k0, s));
			const float2 step = expi2pi_f(phase1(run.stride, s));
			for (int kk = k0; kk < k1; kk++) {
				dst[(run.off + kk) * estride] = z;
				z = cmul(z, step);
			}
		} else {
			double2 z = expi2pi(phase1(run.m0 + run.stride * k0, s));
			const double2 step = expi2pi(phase1(run.stride, s));
			for (int kk = k0; kk < k1; kk++) {
				dst[(run.off + kk) * estride] = to_c<C>(z);
				z = cmul(z, step);
			}
		}
	}
}

// Table indices of a segment's seed: z_0 = prod_e T_e(index_e).
struct SeedIdx {
	int a[3], b[3];   // axis e: entry a[e] (full) or a[e] * b[e] (coarse x fine, b[e] >= 0)
	int w;            // entry of the recurrence step exp(2 pi i s_last)
};

template <int D>
__device__ __forceinline__ SeedIdx seed_index(const TabSpec &sp, const Seg &g)
{
	SeedIdx x;
	int v[3] = {g.p0, g.p1, 0};
	v[D - 1] = g.start;
#pragma unroll
	for (int e = 0; e < D; e++) {
		const int m = v[e] - sp.lo[e];
		if (sp.full[e]) {
			x.a[e] = sp.offc[e] + m;
			x.b[e] = -1;
		} else {
			x.a[e] = sp.offc[e] + (m >> 3);
			x.b[e] = sp.offf[e] + (m & 7);
		}
	}
	x.w = sp.offf[D - 1] + 1;
	return x;
}

template <int D, typename C>
__device__ __forceinline__ C seed_from(const C *row, int estride, const SeedIdx &x)
{
	C z = row[x.a[D - 1] * estride];
	if (x.b[D - 1] >= 0)
		z = cmul(z, row[x.b[D - 1] * estride]);
#pragma unroll
	for (int e = 0; e < D - 1; e++) {
		C t = row[x.a[e] * estride];
		if (x.b[e] >= 0)
			t = cmul(t, row[x.b[e] * estride]);
		z = cmul(z, t);
	}
	return z;
}

// The same from tables in global memory written earlier in the same launch: loads go to L2 (ld.global.cg), never
// to a possibly stale L1 line.
template <int D, typename C>
__device__ __forceinline__ C seed_from_l2(const C *row, size_t estride, const SeedIdx &x)
{
	C z = __ldcg(row + x.a[D - 1] * estride);
	if (x.b[D - 1] >= 0)
		z = cmul(z, __ldcg(row + x.b[D - 1] * estride));
#pragma unroll
	for (int e = 0; e < D - 1; e++) {
		C t = __ldcg(row + x.a[e] * estride);
		if (x.b[e] >= 0)
			t = cmul(t, __ldcg(row + x.b[e] * estride));
		z = cmul(z, t);
	}
	return z;
}

// Cartesian force F = fscale * sum_e g_e b_e and fractional gradient -fscale * 2 pi * g of particle j.
template <int D>
__device__ __forceinline__ void write_force_out(double *F_out, double *gfrac_out, const double *recip, double fscale,
                                                int j, const double *g)
{
	if (F_out) {
#pragma unroll
		for (int c = 0; c < D; c++) {
			double f = 0.0;
#pragma unroll
			for (int e = 0; e < D; e++)
				f = fma(g[e], recip[e * D + c], f);
			F_out[(size_t)j * D + c] = fscale * f;
		}
	}
	if (gfrac_out) {
		const double gs = -fscale * 6.283185307179586476925286766559;
#pragma unroll
		for (int e = 0; e < D; e++)
			gfrac_out[(size_t)j * D + e] = gs * g[e];
	}
}

// An evaluation is skipped when its skip word is nonzero (a finished minimisation) or its stage word differs from the
// launch's stage (the precision schedule of batched minimisations). Both pointers may be null.
__device__ __forceinline__ bool eval_skipped(const int *skip, const int *stage, int want_stage)
{
	return (skip && *(volatile const int *)skip) || (stage && *(volatile const int *)stage != want_stage);
}

// Work queue of a persistent multi-instance launch: q[0] the next item (taken with an atomic add), q[1] the blocks
// that found it empty. The last block to leave resets both, so the next launch starts at item 0. Items write their
// own outputs, so the order in which blocks take them does not change any result.

__device__ __forceinline__ void queue_leave(unsigned *q)
{
	if (threadIdx.x == 0) {
		__threadfence();
		if (atomicAdd(q + 1, 1u) == gridDim.x - 1) {
			q[0] = 0u;
			q[1] = 0u;
		}
	}
}

// Instance of a multi-instance launch's block: pre[b] <= item < pre[b + 1] (binary search, B + 1 prefix sums).
__device__ __forceinline__ int find_instance(const int *pre, int B, int item)
{
	int lo = 0, hi = B;
	while (hi - lo > 1) {
		const int mid = (lo + hi) >> 1;
		if (__ldg(pre + mid) <= item)
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

constexpr int kForceUChunk = 128;   // segments whose slot weights are staged in shared memory at once

// Block-shared scalars and small arrays of the rho / reduce / force bodies. They live in ONE shared variable of a
// non-template function, so a kernel that inlines several bodies (every dimension and precision of the fused batch
// kernel) holds one set per block instead of one per body instantiation.
struct BodyShared {
	TabSpec sp;
	Seg seg[kForceUChunk];
	double2 red[8][32];
	double pos[32 * 3];   // the force block's particles' coordinates (loaded together with its table spec)
	int last;
};
__device__ __forceinline__ BodyShared &body_shared()
{
	__shared__ BodyShared s;
	return s;
}

// Bounded wait of a whole block until *ready >= need (a count other blocks of the same launch raise after their
// items' results are visible). Thread 0 polls; after kReadySpins polls it sets *err and gives up, so a fault ends the
// launch with an error status instead of a hang.
constexpr unsigned kReadySpins = 1u << 22;
__device__ __forceinline__ void wait_ready(const unsigned *ready, unsigned need, unsigned *err, unsigned spins)
{
	if (threadIdx.x == 0) {
		const unsigned limit = spins ? spins : kReadySpins;
		unsigned it = 0;
		while (*(volatile const unsigned *)ready < need) {
			if (++it > limit) {
				atomicExch(err, 1u);
				break;
			}
			__nanosleep(32);
		}
		__threadfence();
	}
	__syncthreads();
}

// The stage test and the bounded wait of one body call. The three-kernel launches pass their arguments' stage words
// and no wait; the fused batch launch sets them per item, so that its bodies read the instances' descriptors from
// global memory as they are and keep no modified copy in registers.
struct ItemCtl {
	const int *stage;
	int want_stage;
	// wait until *ready >= ready_need (the instance's items of the previous phase done) before reading their results;
	// err is raised when that bounded wait runs out (after ready_spins polls, 0: kReadySpins). Null: no wait.
	const unsigned *ready = nullptr;
	unsigned ready_need = 0, ready_spins = 0;
	unsigned *err = nullptr;
};

// ---------------------------------------------------------------------------------------------------------------
// rho pass
// ---------------------------------------------------------------------------------------------------------------
struct RhoArgs {
	const double *frac;       // N x D fractional coordinates
	int N;
	int per_split;            // particles per block (blockIdx.y)
	int chunk;                // particles whose tables are staged at once
	const Seg *segs;          // ngroups * 32 (padding segments have len 0)
	const int *bstart;        // nbgroups + 1: rho groups (warps) of each block group
	const TabSpec *bspec;     // nbgroups
	int nseg, nslot;          // nseg = ngroups * 32, nslot = nseg * L
	double2 *partial;         // [nsplit / cluster][nslot]
	const int *skip;          // if not null and nonzero, the launch does nothing (a finished minimisation)
	const int *stage;         // if not null, the launch does nothing unless *stage == want_stage
	int want_stage;
	double *frac_copy;        // if not null, the blocks of block group 0 also store their particles' coordinates
	                          // there (frac is then host memory the kernels that follow do not read)
	int early;                // nonzero: frac was complete before the previous kernel on the stream was enqueued and
	                          // nothing in flight writes it, so the blocks run their main loop before waiting for
	                          // that kernel (skip, stage and frac_copy are then null)
};

constexpr int kRhoWarps = 8;
constexpr int kRhoThreads = kRhoWarps * 32;

// Grid (nbgroups, nsplit), clusters of `csize` blocks along y (the particle splits of one block group). Warp w of a
// block owns the 32 segments of rho group bstart[g] + w (one per lane) and walks every particle of the block's split;
// the tables of a chunk of particles are built once for the block group's spec and shared by all warps. The cluster's
// blocks are added in rank order through distributed shared memory into one partial row.
// Block (bg, split) of the rho pass. CLUSTER: the blocks of a thread-block cluster (consecutive splits) are added
// through distributed shared memory into partial row split / cluster size; otherwise the block writes row `split`.
template <int D, int L, bool MIXED, bool CLUSTER>
__device__ __forceinline__ void rho_body(const RhoArgs &a, const int bg, const int split, const ItemCtl ctl)
{
	typedef typename std::conditional<MIXED, float2, double2>::type C;
	constexpr int SUB = 16;
	extern __shared__ __align__(16) unsigned char smem[];
	C *tab = reinterpret_cast<C *>(smem);             // chunk x row (particle-major)
	double2 *red = reinterpret_cast<double2 *>(smem); // after the loop: kRhoWarps x L x 32
	TabSpec &sp = body_shared().sp;

	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (threadIdx.x == 0)
		sp = a.bspec[bg];
	const int g0 = a.bstart[bg], nwg = a.bstart[bg + 1] - g0;
	const bool active = warp < nwg;
	const int q = (g0 + (active ? warp : 0)) * 32 + lane;
	const Seg sg = a.segs[q];
	const int j0 = min(a.N, split * a.per_split);
	const int j1 = min(a.N, j0 + a.per_split);
	// inputs of this step are complete (programmatic dependent launch); with a.early only the partial rows wait
	if (!a.early)
		cudaGridDependencySynchronize();
	if (eval_skipped(a.skip, ctl.stage, ctl.want_stage))   // uniform over the instance: no block reaches a cluster barrier
		return;
	if (a.frac_copy && bg == 0)
		for (int t = threadIdx.x; t < (j1 - j0) * D; t += kRhoThreads)
			a.frac_copy[(size_t)j0 * D + t] = a.frac[(size_t)j0 * D + t];
	__syncthreads();
	const int row = sp.row | 1;        // odd row stride: consecutive particles' rows start in different banks
	SeedIdx ix = seed_index<D>(sp, sg);
	if (sg.len == 0 || !active) {
		// padding lanes read entry 0 of every table (always present)
#pragma unroll
		for (int e = 0; e < 3; e++) {
			ix.a[e] = 0;
			ix.b[e] = -1;
		}
	}

	// per-slot sums in the compute type (FP32 in the mixed path, flushed into the FP64 acc every SUB particles)
	typedef typename std::conditional<MIXED, float, double>::type R;
	double2 acc[L];
	C accC[L];
#pragma unroll
	for (int r = 0; r < L; r++) {
		acc[r] = make_double2(0.0, 0.0);
		accC[r].x = 0;
		accC[r].y = 0;
	}
	int since_flush = 0;

	for (int cj = j0; cj < j1; cj += a.chunk) {
		const int cnt = min(a.chunk, j1 - cj);
		if (cj != j0)
			__syncthreads();
		build_tables<D, C>(sp, a.frac, cj, cnt, cnt, tab, row, 1, threadIdx.x, kRhoThreads);
		__syncthreads();
		if (!active)
			continue;
		int i = 0;
		for (; i + 1 < cnt; i += 2) {
			const C *r0 = tab + i * row, *r1 = r0 + row;
			C z0 = seed_from<D, C>(r0, 1, ix), z1 = seed_from<D, C>(r1, 1, ix);
			const C w0 = r0[ix.w], w1 = r1[ix.w];
			// three-term recurrence along the segment
			const R c0 = (R)2 * w0.x, c1 = (R)2 * w1.x;
			C p0 = z0, p1 = z1, q0 = cmul(z0, w0), q1 = cmul(z1, w1);
			acc_add(accC[0], p0, p1);
			acc_add(accC[1], q0, q1);
			if constexpr (MIXED) {
				// sign-free form: accC[r] holds s_r times the slot's sum
				const float2 c0p = make_float2(c0, c0), c0n = make_float2(-c0, -c0);
				const float2 c1p = make_float2(c1, c1), c1n = make_float2(-c1, -c1);
#pragma unroll
				for (int r = 2; r < L; r++) {
					const float2 n0 = seg_next(r, c0p, c0n, q0, p0), n1 = seg_next(r, c1p, c1n, q1, p1);
					acc_add(accC[r], n0, n1);
					p0 = q0;
					q0 = n0;
					p1 = q1;
					q1 = n1;
				}
			} else {
#pragma unroll
				for (int r = 2; r < L; r++) {
					const C n0 = cheb_next(c0, q0, p0), n1 = cheb_next(c1, q1, p1);
					acc_add(accC[r], n0, n1);
					p0 = q0;
					q0 = n0;
					p1 = q1;
					q1 = n1;
				}
			}
			if (MIXED && (since_flush += 2) >= SUB) {
				since_flush = 0;
#pragma unroll
				for (int r = 0; r < L; r++) {
					const double sg = slot_negated(r) ? -1.0 : 1.0;
					acc[r].x += sg * (double)accC[r].x;
					acc[r].y += sg * (double)accC[r].y;
					accC[r].x = 0;
					accC[r].y = 0;
				}
			}
		}
		if (i < cnt) {
			const C *r0 = tab + i * row;
			C z0 = seed_from<D, C>(r0, 1, ix);
			const C w0 = r0[ix.w];
			const R c0 = (R)2 * w0.x;
			C p0 = z0, q0 = cmul(z0, w0);
			acc_add(accC[0], p0);
			acc_add(accC[1], q0);
			if constexpr (MIXED) {
				const float2 c0p = make_float2(c0, c0), c0n = make_float2(-c0, -c0);
#pragma unroll
				for (int r = 2; r < L; r++) {
					const float2 n0 = seg_next(r, c0p, c0n, q0, p0);
					acc_add(accC[r], n0);
					p0 = q0;
					q0 = n0;
				}
			} else {
#pragma unroll
				for (int r = 2; r < L; r++) {
					const C n0 = cheb_next(c0, q0, p0);
					acc_add(accC[r], n0);
					p0 = q0;
					q0 = n0;
				}
			}
		}
	}
#pragma unroll
	for (int r = 0; r < L; r++) {
		if (MIXED) {
			const double sg = slot_negated(r) ? -1.0 : 1.0;
			acc[r].x += sg * (double)accC[r].x;
			acc[r].y += sg * (double)accC[r].y;
		} else {
			acc[r].x = (double)accC[r].x;
			acc[r].y = (double)accC[r].y;
		}
	}
	// Early mode: the sums above read only positions and the k-set; the partial rows below are still read by the
	// previous evaluation's reduce kernel until the previous kernel on the stream has completed.
	if (a.early)
		cudaGridDependencySynchronize();
	cudaTriggerProgrammaticLaunchCompletion();   // the next kernel may be scheduled; it waits for this grid

	if constexpr (!CLUSTER) {
		// one partial row per block
		if (active) {
#pragma unroll
			for (int r = 0; r < L; r++)
				a.partial[(size_t)split * a.nslot + (size_t)r * a.nseg + (g0 + warp) * 32 + lane] = acc[r];
		}
		return;
	}
	// this block's sums, layout [warp][r][lane], then the cluster's blocks in rank order
	cg::cluster_group cluster = cg::this_cluster();
	__syncthreads();
	if (active) {
#pragma unroll
		for (int r = 0; r < L; r++)
			red[(warp * L + r) * 32 + lane] = acc[r];
	}
	cluster.sync();
	const int cs = (int)cluster.num_blocks();
	const int rank = (int)cluster.block_rank();
	const int total = nwg * L * 32;
	const int per = (total + cs - 1) / cs;
	const size_t out_row = (size_t)(split / cs) * a.nslot;
	for (int e = rank * per + threadIdx.x; e < min(total, (rank + 1) * per); e += kRhoThreads) {
		const int w = e / (L * 32), r = (e / 32) % L, ln = e & 31;
		// the cluster's (at most 8) values are loaded together, then added in rank order
		double2 v[8];
#pragma unroll
		for (int k = 0; k < 8; k++)
			if (k < cs)
				v[k] = cluster.map_shared_rank(red, k)[e];
		double2 t = make_double2(0.0, 0.0);
#pragma unroll
		for (int k = 0; k < 8; k++)
			if (k < cs) {
				t.x += v[k].x;
				t.y += v[k].y;
			}
		a.partial[out_row + (size_t)r * a.nseg + (g0 + w) * 32 + ln] = t;
	}
	cluster.sync();
}

// Grid (nbgroups, nsplit), clusters of `csize` blocks along y (the particle splits of one block group). Warp w of a
// block owns the 32 segments of rho group bstart[g] + w (one per lane) and walks every particle of the block's split;
// the tables of a chunk of particles are built once for the block group's spec and shared by all warps. The cluster's
// blocks are added in rank order through distributed shared memory into one partial row.
template <int D, int L, bool MIXED>
__global__ void __launch_bounds__(kRhoThreads, 3) cc_rho_kernel(RhoArgs a)
{
	rho_body<D, L, MIXED, true>(a, blockIdx.x, blockIdx.y, ItemCtl{a.stage, a.want_stage});
}

// ---------------------------------------------------------------------------------------------------------------
// split reduction, u = V conj(rho), energy
// ---------------------------------------------------------------------------------------------------------------
struct ReduceArgs {
	const double2 *partial;   // [nsplit][nslot]
	int nsplit, nslot;
	const double *slotV;
	double rho_offset;        // added to Re rho of every slot
	double2 *rho_slot, *u_slot;
	double *eblock;           // [gridDim.x]
	unsigned *ticket;         // 1, zero between launches
	double inv_vol, shift;
	double *E_out;
	int finalize;             // 0: the force kernel that follows sums eblock into E_out
	const int *skip;
	const int *stage;
	int want_stage;
	// S2 form (the reference's ShiftedCCPotential_S2) when not null: targets S0 per slot, e = V (|rho|^2 / N - S0)^2,
	// u = V (|rho|^2 / N - S0) conj(rho); npart = N
	const double *slotS0;
	double npart;
};

constexpr int kRedThreads = 256;   // 32 slots x 8 split chunks

// Block `chunk` (32 slots) of the split reduction of an instance with `nchunks` such blocks.
__device__ __forceinline__ void reduce_body(const ReduceArgs &a, const int chunk, const int nchunks)
{
	double2 (&sh)[8][32] = body_shared().red;
	int &sh_last = body_shared().last;
	const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
	const int slot = chunk * 32 + lane;
	const int per = (a.nsplit + 7) >> 3;
	cudaGridDependencySynchronize();
	cudaTriggerProgrammaticLaunchCompletion();
	if (eval_skipped(a.skip, a.stage, a.want_stage))
		return;
	const int s0 = min(a.nsplit, c * per), s1 = min(a.nsplit, s0 + per);
	double2 t = make_double2(0.0, 0.0);
	if (slot < a.nslot) {
		int sp = s0;
		for (; sp + 4 <= s1; sp += 4) {
			const double2 v0 = __ldcg(&a.partial[(size_t)sp * a.nslot + slot]);
			const double2 v1 = __ldcg(&a.partial[(size_t)(sp + 1) * a.nslot + slot]);
			const double2 v2 = __ldcg(&a.partial[(size_t)(sp + 2) * a.nslot + slot]);
			const double2 v3 = __ldcg(&a.partial[(size_t)(sp + 3) * a.nslot + slot]);
			t.x += v0.x;
			t.y += v0.y;
			t.x += v1.x;
			t.y += v1.y;
			t.x += v2.x;
			t.y += v2.y;
			t.x += v3.x;
			t.y += v3.y;
		}
		for (; sp < s1; sp++) {
			const double2 v = __ldcg(&a.partial[(size_t)sp * a.nslot + slot]);
			t.x += v.x;
			t.y += v.y;
		}
	}
	sh[c][lane] = t;
	__syncthreads();
	if (c == 0) {
		double2 rho = sh[0][lane];
#pragma unroll
		for (int k = 1; k < 8; k++) {
			rho.x += sh[k][lane].x;
			rho.y += sh[k][lane].y;
		}
		double e = 0.0;
		if (slot < a.nslot) {
			rho.x += a.rho_offset;
			a.rho_slot[slot] = rho;
			double v = a.slotV[slot];
			const double r2 = rho.x * rho.x + rho.y * rho.y;
			if (a.slotS0) {
				const double ds = r2 / a.npart - a.slotS0[slot];
				v *= ds;
				e = v * ds;
			} else {
				e = v * r2;
			}
			a.u_slot[slot] = make_double2(v * rho.x, -v * rho.y);
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
			e += __shfl_down_sync(0xffffffffu, e, o);
		if (lane == 0)
			a.eblock[chunk] = e;
	}
	if (!a.finalize)
		return;
	__threadfence();
	__syncthreads();
	if (threadIdx.x == 0)
		sh_last = (atomicAdd(a.ticket, 1u) == (unsigned)nchunks - 1);
	__syncthreads();
	if (!sh_last || c != 0)
		return;
	__threadfence();
	double e = 0.0;
	for (int b = lane; b < nchunks; b += 32)
		e += __ldcg(&a.eblock[b]);
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		e += __shfl_down_sync(0xffffffffu, e, o);
	if (lane == 0) {
		*a.E_out = e * a.inv_vol + a.shift;
		*a.ticket = 0u;
	}
}

// Item `item` (kWideSlots slots, one per thread) of the split reduction in the fused batch launch: every slot sums the
// partial rows in row order, then the block's energy terms are added (lanes by a fixed tree, warps in order) into
// eblock[item]. Wider than reduce_body's 32-slot chunks so that a batch's many small reductions cost few work items;
// for up to 8 partial rows the sums equal reduce_body's bitwise (its 8 row chunks then hold one row each).
constexpr int kWideSlots = 256;
__device__ __forceinline__ void reduce_body_wide(const ReduceArgs &a, const int item, const ItemCtl ctl)
{
	double2(&sh)[8][32] = body_shared().red;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	cudaGridDependencySynchronize();
	cudaTriggerProgrammaticLaunchCompletion();
	// The wait comes first, also for a skipped instance: its last force item resets the instance's counts, which must
	// not happen while one of its rho or reduce items is still to be counted.
	if (ctl.ready)
		wait_ready(ctl.ready, ctl.ready_need, ctl.err, ctl.ready_spins);
	if (eval_skipped(a.skip, ctl.stage, ctl.want_stage))
		return;
	const int slot = item * kWideSlots + threadIdx.x;
	double e = 0.0;
	if (slot < a.nslot) {
		double2 t = make_double2(0.0, 0.0);
		int sp = 0;
		for (; sp + 4 <= a.nsplit; sp += 4) {
			const double2 v0 = __ldcg(&a.partial[(size_t)sp * a.nslot + slot]);
			const double2 v1 = __ldcg(&a.partial[(size_t)(sp + 1) * a.nslot + slot]);
			const double2 v2 = __ldcg(&a.partial[(size_t)(sp + 2) * a.nslot + slot]);
			const double2 v3 = __ldcg(&a.partial[(size_t)(sp + 3) * a.nslot + slot]);
			t.x += v0.x;
			t.y += v0.y;
			t.x += v1.x;
			t.y += v1.y;
			t.x += v2.x;
			t.y += v2.y;
			t.x += v3.x;
			t.y += v3.y;
		}
		for (; sp < a.nsplit; sp++) {
			const double2 v = __ldcg(&a.partial[(size_t)sp * a.nslot + slot]);
			t.x += v.x;
			t.y += v.y;
		}
		t.x += a.rho_offset;
		a.rho_slot[slot] = t;
		double v = a.slotV[slot];
		const double r2 = t.x * t.x + t.y * t.y;
		if (a.slotS0) {
			const double ds = r2 / a.npart - a.slotS0[slot];
			v *= ds;
			e = v * ds;
		} else {
			e = v * r2;
		}
		a.u_slot[slot] = make_double2(v * t.x, -v * t.y);
	}
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		e += __shfl_down_sync(0xffffffffu, e, o);
	if (lane == 0)
		sh[0][warp].x = e;
	__syncthreads();
	if (threadIdx.x == 0) {
		double b = 0.0;
		for (int w = 0; w < kRhoWarps; w++)
			b += sh[0][w].x;
		a.eblock[item] = b;
	}
}

static __global__ void __launch_bounds__(kRedThreads) cc_reduce_kernel(ReduceArgs a)
{
	reduce_body(a, blockIdx.x, gridDim.x);
}

// rho in input-mode order (repeated modes read their shared slot)
static __global__ void cc_gather_rho_kernel(const double2 *__restrict__ rho_slot, const int *__restrict__ mode_slot, int M,
                                     double2 *__restrict__ rho_mode)
{
	const int m = blockIdx.x * blockDim.x + threadIdx.x;
	if (m < M)
		rho_mode[m] = rho_slot[mode_slot[m]];
}

// E = shift when there is no constraint
static __global__ void cc_set_scalar_kernel(double *p, double v) { *p = v; }

// n doubles from src (mapped pinned host memory) to dst (device memory)
static __global__ void cc_upload_kernel(const double *__restrict__ src, double *__restrict__ dst, int64_t n)
{
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n)
		dst[i] = src[i];
}

// ---------------------------------------------------------------------------------------------------------------
// force pass
// ---------------------------------------------------------------------------------------------------------------
struct ForceArgs {
	const double *frac;       // N x D
	int N;
	const Seg *segs;
	const int *kstart;        // nksplit + 1: segment range of each split
	const TabSpec *kspec;     // nksplit
	int nksplit;
	const double2 *u_slot;    // [nslot], slot of (segment q, step r) = r * nseg + q
	int nseg;
	double *partialG;         // [nksplit][N][D], only for nksplit > 1
	unsigned *counters;       // [ceil(N/32)], zero between launches
	double recip[9];          // reciprocal basis, row e = b_e (Cartesian)
	double fscale;            // 2 / Volume
	double *F_out;            // N x D Cartesian forces, or nullptr
	double *gfrac_out;        // N x D dPhi/ds, or nullptr
	const double *eblock;     // energy partials of the reduce blocks (neblock), summed into E_out by block (0, 0) when
	int neblock;              // E_out is set (the reduce kernel then leaves E to this kernel)
	double inv_vol, shift;
	double *E_out;
	const int *skip;
	const int *stage;
	int want_stage;
};

constexpr int kForceWarps = 8;
constexpr int kForceThreads = kForceWarps * 32;

template <int D>
__device__ __forceinline__ void write_force(const ForceArgs &a, int j, const double *g)
{
	write_force_out<D>(a.F_out, a.gfrac_out, a.recip, a.fscale, j, g);
}

constexpr int kForceRun = 4;        // FP64 force pass: segments of a lattice line on one recurrence before a new seed
// The same in the mixed path (FP32 recurrences). Measured at 2D N=1e5 chi=0.2 against the reference's FP64 forces:
// runs of 1 / 2 / 4 segments give 1.0e-6 / 1.8e-6 / 7.9e-6 of max |F| (the energy is unchanged, 7e-9 relative) and a
// 3.59 / 3.56 / 3.42 ms evaluation.
constexpr int kForceRunMixed = 4;

// Dynamic shared memory of the force kernel for tables of `row` entries: the staged weights, then the tables; the
// per-warp sums reuse it after the loop.
template <typename C> __host__ __device__ constexpr size_t force_smem_bytes(int row, int d, int L)
{
	return ((size_t)L * kForceUChunk + (size_t)row * 32) * sizeof(C) > (size_t)kForceWarps * 32 * d * sizeof(double)
	           ? ((size_t)L * kForceUChunk + (size_t)row * 32) * sizeof(C)
	           : (size_t)kForceWarps * 32 * d * sizeof(double);
}

// Grid (ceil(N/32), nksplit). Block = 32 particles (lanes) x 8 warps, each warp on a contiguous run of the split's
// segments; the tables of the block's particles for the split are built once (entry-major, so a warp reads 32
// consecutive entries). The slot weights u of up to kForceUChunk segments at a time are staged in shared memory in the
// compute type (a warp's read of one weight is a broadcast): FP64 slot-major, mixed segment-major with each pair of
// components swapped and signed for the sign-free FP32 recurrence.
template <int D, int L, bool MIXED>
__device__ __forceinline__ void force_body(const ForceArgs &a, const int pgroup, const int ks, const ItemCtl ctl)
{
	typedef typename std::conditional<MIXED, float, double>::type R;
	typedef typename std::conditional<MIXED, float2, double2>::type C;
	extern __shared__ __align__(16) unsigned char smem[];
	C *sh_u = reinterpret_cast<C *>(smem);           // L x kForceUChunk, slot-major
	C *tab = sh_u + L * kForceUChunk;                // row x 32, entry-major
	double *sh_g = reinterpret_cast<double *>(smem); // reused after the loop: kForceWarps x 32 x D
	TabSpec &sp = body_shared().sp;
	Seg *sh_seg = body_shared().seg;
	int &sh_last = body_shared().last;

	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int pbase = pgroup * 32;
	const int j = pbase + lane;
	const int nvalid = min(32, a.N - pbase);
	const int q0 = a.kstart[ks], q1 = a.kstart[ks + 1];
	// The skip and stage words are written by kernels that completed before this evaluation's rho pass (whose
	// completion this block's launch implies), like the positions: a finished instance builds no tables. In the fused
	// batch launch its force items still wait for its reduce items (which waited for its rho items), so that the last
	// of them resets the instance's counts only once every item of the instance has been counted.
	if (eval_skipped(a.skip, ctl.stage, ctl.want_stage)) {
		if (ctl.ready)
			wait_ready(ctl.ready, ctl.ready_need, ctl.err, ctl.ready_spins);
		return;
	}
	// the spec and the block's coordinates are loaded together (neither waits for the other)
	double *pos = body_shared().pos;
	if (threadIdx.x == 0)
		sp = a.kspec[ks];
	for (int t = threadIdx.x; t < nvalid * D; t += kForceThreads)
		pos[t] = a.frac[(size_t)pbase * D + t];
	__syncthreads();
	// The tables need only the positions, which the rho pass of this evaluation has already read: they are built
	// while the reduce kernel still runs (programmatic dependent launch), before waiting for u.
	build_tables<D, C>(sp, pos, 0, 32, nvalid, tab, 1, 32, threadIdx.x, kForceThreads);
	cudaGridDependencySynchronize();   // u of this step is complete
	if (ctl.ready)
		wait_ready(ctl.ready, ctl.ready_need, ctl.err, ctl.ready_spins);
	if (eval_skipped(a.skip, ctl.stage, ctl.want_stage))   // uniform over the instance
		return;
	if (a.E_out && pgroup == 0 && ks == 0 && warp == 0) {
		// the energy, summed in the order of the reduce kernel's last block
		double e = 0.0;
		for (int b = lane; b < a.neblock; b += 32)
			e += __ldcg(a.eblock + b);
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
			e += __shfl_down_sync(0xffffffffu, e, o);
		if (lane == 0)
			*a.E_out = e * a.inv_vol + a.shift;
	}

	double g[D];
#pragma unroll
	for (int e = 0; e < D; e++)
		g[e] = 0.0;
	for (int c0 = q0; c0 < q1; c0 += kForceUChunk) {
		const int nq = min(kForceUChunk, q1 - c0);
		__syncthreads();   // tables complete (first chunk); the previous chunk's weights are no longer read
		// FP64: slot-major (a warp's read of one weight is a broadcast); mixed: segment-major, a segment's 8 FP32
		// weights contiguous (read as four 16-byte broadcasts)
		// weights, mixed: (s_r u.y, s_r u.x) in FP32 for the sign-free recurrence's y_r = s_r z_r, so that the packed
		// product with y_r is (u.y z.x, u.x z.y), whose sum is Im(u z)
		for (int e = threadIdx.x; e < nq * L; e += kForceThreads) {
			const int r = e / nq, qq = e - r * nq;
			const double2 u = __ldcg(a.u_slot + (size_t)r * a.nseg + c0 + qq);
			if constexpr (MIXED) {
				const float sg = slot_negated(r) ? -1.0f : 1.0f;
				sh_u[qq * L + r] = make_float2(sg * (float)u.y, sg * (float)u.x);
			} else {
				sh_u[r * kForceUChunk + qq] = u;
			}
		}
		for (int e = threadIdx.x; e < nq; e += kForceThreads) {
			sh_seg[e] = a.segs[c0 + e];
		}
		__syncthreads();
		if constexpr (!MIXED) {
			// FP64: warp w takes a contiguous run of the chunk's segments; a segment that continues the previous one
			// on its lattice line (same line, start + L, previous one full) continues the three-term recurrence
			// instead of being seeded from the tables, for up to kForceRun segments in a row
			const int per = (nq + kForceWarps - 1) / kForceWarps;
			const int qa = min(nq, warp * per), qb = min(nq, qa + per);
			double2 p = make_double2(0.0, 0.0), q = make_double2(0.0, 0.0);
			double c = 0.0;
			int run = 0;
			Seg prev = {0, 0, 0, 0};
			for (int qq = qa; qq < qb; qq++) {
				const Seg sgm = sh_seg[qq];
				if (sgm.len == 0) {   // padding segment of a rho group: weight 0, no table entries
					run = 0;
					continue;
				}
				const double2 *uu = sh_u + qq;
				double2 z0, z1;
				if (run > 0 && run < kForceRun && prev.len == L && sgm.p0 == prev.p0 && sgm.p1 == prev.p1 &&
				    sgm.start == prev.start + L) {
					z0 = cheb_next(c, q, p);
					z1 = cheb_next(c, z0, q);
					run++;
				} else {
					const SeedIdx ix = seed_index<D>(sp, sgm);
					z0 = seed_from<D, double2>(tab + lane, 32, ix);
					const double2 w = tab[ix.w * 32 + lane];
					c = 2.0 * w.x;
					z1 = cmul(z0, w);
					run = 1;
				}
				const double2 u0 = uu[0], u1 = uu[kForceUChunk];
				double S0 = u0.x * z0.y + u0.y * z0.x, S1;
				{
					const double t = u1.x * z1.y + u1.y * z1.x;
					S0 += t;
					S1 = t;
				}
				p = z0;
				q = z1;
#pragma unroll
				for (int r = 2; r < L; r++) {
					const double2 n = cheb_next(c, q, p);
					const double2 u = uu[r * kForceUChunk];
					const double t = u.x * n.y + u.y * n.x;
					S0 += t;
					S1 = fma((double)r, t, S1);
					p = q;
					q = n;
				}
				if (D >= 2)
					g[0] = fma(S0, (double)sgm.p0, g[0]);
				if (D >= 3)
					g[1] = fma(S0, (double)sgm.p1, g[1]);
				g[D - 1] = fma(S0, (double)sgm.start, g[D - 1] + S1);
				prev = sgm;
			}
		} else {
			// the chunk's (at most kForceUChunk / kForceWarps) segment terms of each gradient component are added in
			// FP32 and leave FP32 once per chunk
			float gf[D];
#pragma unroll
			for (int e = 0; e < D; e++)
				gf[e] = 0.0f;
			// as in FP64, warp w takes a contiguous run of the chunk's segments, and a segment that continues the
			// previous one on its lattice line continues the (sign-free) recurrence, here for up to kForceRunMixed
			// segments in a row; the sign pattern s_r and the coefficients' signs have period 4, which divides L, so
			// the continuation's slots 0 and 1 are steps L and L + 1 of the same recurrence
			const int per = (nq + kForceWarps - 1) / kForceWarps;
			const int qa = min(nq, warp * per), qb = min(nq, qa + per);
			float2 p = make_float2(0.0f, 0.0f), q = p, cp = p, cn = p;
			int run = 0;
			Seg prev = {0, 0, 0, 0};
			for (int qq = qa; qq < qb; qq++) {
				const Seg sgm = sh_seg[qq];
				if (sgm.len == 0) {   // padding segment of a rho group: weight 0, no table entries
					run = 0;
					continue;
				}
				const float4 *uu = reinterpret_cast<const float4 *>(sh_u + qq * L);   // slot pairs (2r, 2r + 1)
				// packed FP32x2: A = sum_r P_r and B = sum_r r P_r of the products P_r = (s_r u_r) * y_r, whose two
				// components add up to Im(u_r z_r)
				float2 y0, y1;
				if (run > 0 && run < kForceRunMixed && prev.len == L && sgm.p0 == prev.p0 && sgm.p1 == prev.p1 &&
				    sgm.start == prev.start + L) {
					y0 = seg_next(L, cp, cn, q, p);
					y1 = seg_next(L + 1, cp, cn, y0, q);
					run++;
				} else {
					const SeedIdx ix = seed_index<D>(sp, sgm);
					const C z = seed_from<D, C>(tab + lane, 32, ix);
					const C w = tab[ix.w * 32 + lane];
					const float c = 2.0f * w.x;
					cp = make_float2(c, c);
					cn = make_float2(-c, -c);
					y0 = z;
					y1 = cmul(z, w);
					run = 1;
				}
				p = y0;
				q = y1;
				const float4 u01 = uu[0];
				float2 A = __fmul2_rn(make_float2(u01.x, u01.y), p);
				float2 B = __fmul2_rn(make_float2(u01.z, u01.w), q);
				A = __fadd2_rn(A, B);
#pragma unroll
				for (int r = 2; r < L; r += 2) {
					const float4 uv = uu[r / 2];
					const float2 n = seg_next(r, cp, cn, q, p);
					const float2 P = __fmul2_rn(make_float2(uv.x, uv.y), n);
					A = __fadd2_rn(A, P);
					B = __ffma2_rn(make_float2((float)r, (float)r), P, B);
					const float2 n2 = seg_next(r + 1, cp, cn, n, q);
					const float2 P2 = __fmul2_rn(make_float2(uv.z, uv.w), n2);
					A = __fadd2_rn(A, P2);
					B = __ffma2_rn(make_float2((float)(r + 1), (float)(r + 1)), P2, B);
					p = n;
					q = n2;
				}
				const float S0 = A.x + A.y, S1 = B.x + B.y;
				if (D >= 2)
					gf[0] = fmaf(S0, (float)sgm.p0, gf[0]);
				if (D >= 3)
					gf[1] = fmaf(S0, (float)sgm.p1, gf[1]);
				gf[D - 1] = fmaf(S0, (float)sgm.start, gf[D - 1] + S1);
				prev = sgm;
			}
#pragma unroll
			for (int e = 0; e < D; e++)
				g[e] += (double)gf[e];
		}
	}

	cudaTriggerProgrammaticLaunchCompletion();
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
		for (int w2 = 1; w2 < kForceWarps; w2++)
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
		sh_last = (atomicAdd(&a.counters[pgroup], 1u) == (unsigned)(a.nksplit - 1));
	__syncwarp();
	if (!sh_last)
		return;
	__threadfence();
	if (j < a.N) {
		double v[D];
#pragma unroll
		for (int e = 0; e < D; e++)
			v[e] = __ldcg(&a.partialG[(size_t)j * D + e]);
		for (int k2 = 1; k2 < a.nksplit; k2++)
#pragma unroll
			for (int e = 0; e < D; e++)
				v[e] += __ldcg(&a.partialG[((size_t)k2 * a.N + j) * D + e]);
		write_force<D>(a, j, v);
	}
	if (lane == 0)
		a.counters[pgroup] = 0u;
}

template <int D, int L, bool MIXED>
__global__ void __launch_bounds__(kForceThreads, MIXED ? 4 : 3) cc_force_kernel(ForceArgs a)
{
	force_body<D, L, MIXED>(a, blockIdx.x, blockIdx.y, ItemCtl{a.stage, a.want_stage});
}

// ---------------------------------------------------------------------------------------------------------------
// fused batch evaluation: ONE persistent launch per batched energy + gradient step
// ---------------------------------------------------------------------------------------------------------------
// The rho, split-reduction and force items of every instance of a batch (every dimension) come from one work queue,
// in this order: items [0, total[0]) are the rho blocks of every instance, then instance by instance its reduce chunks
// followed by its force blocks (instances by decreasing work). An item raises its instance's count of that phase
// when its results are visible; a reduce item waits (bounded) for its instance's rho count, a force item for its
// reduce count, after building its tables. An item only waits for items taken from the queue before it, by blocks that
// are running and never wait for later items, so the launch cannot deadlock whatever number of blocks is resident. The
// last force item of an instance resets its counts for the next launch. Each instance keeps its own plan, tiles and
// fixed-order sums, so its results are those of the three-kernel batch evaluation, bitwise.
struct MBatchArgs {
	const RhoArgs *rho;
	const ReduceArgs *red;
	const ForceArgs *force;
	const int *dim;       // B: dimension of each instance (1..3)
	const int *pre;       // 4 x (B + 1): prefix sums of each instance's rho, reduce, force, and reduce + force items
	const int *shape;     // 3 x B: rho block groups, reduce chunks, force particle groups
	int B;
	int total[3];
	int want_stage;       // MODE 0 / 1: instances whose stage word differs are skipped (as the three-kernel launches)
	unsigned *queue;      // 2 words, zero between launches
	unsigned *count;      // 3 x B completed items per instance and phase (zero between launches), then 1 error word
	unsigned spins;       // polls of each bounded wait before it gives up (0: kReadySpins)
	unsigned phantom;     // test hook: instance 0's reduce items wait for this many rho items more than it has
};

constexpr int kMBatchThreads = 256;

// The fused batch kernel's current descriptor, copied into shared memory by the whole block at once (one round trip
// to L2 for all its fields, instead of one per field as a body reads them, or a register copy that spills). One
// variable of a non-template function, so the kernel holds one per block.
union ItemDesc {
	RhoArgs rho;
	ReduceArgs red;
	ForceArgs force;
};
__device__ __forceinline__ ItemDesc &item_desc()
{
	__shared__ ItemDesc s;
	return s;
}
// (the previous item's body no longer reads the copy: every item ends at a block barrier)
template <typename T> __device__ __forceinline__ const T &stage_desc(const T *src, T &dst)
{
	static_assert(sizeof(T) % 8 == 0 && alignof(T) >= 8, "descriptors are copied as 8-byte words");
	const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
	unsigned long long *d = reinterpret_cast<unsigned long long *>(&dst);
	for (int t = threadIdx.x; t < (int)(sizeof(T) / 8); t += blockDim.x)
		d[t] = __ldg(s + t);
	__syncthreads();
	return dst;
}

template <int D, int MODE>
__device__ __forceinline__ void mbatch_item(const MBatchArgs &A, int phase, int b, int local)
{
	// MODE 0: FP64, 1: mixed, 2: each instance at the precision of its stage word (mixed while it is 0). The
	// instance's descriptor is read from its copy in shared memory; the stage test and the waits come from `ctl`.
	ItemCtl ctl;
	ctl.err = A.count + 3 * A.B;
	ctl.ready_spins = A.spins;
	ctl.want_stage = A.want_stage;
	if (phase == 0) {
		const RhoArgs &r = stage_desc(A.rho + b, item_desc().rho);
		const int *stage = r.stage;
		const bool mixed = MODE == 1 || (MODE == 2 && stage && *(volatile const int *)stage == 0);
		ctl.stage = MODE == 2 ? nullptr : stage;
		const int ng = __ldg(A.shape + b);
		if constexpr (MODE != 0) {
			if (mixed) {
				rho_body<D, 8, true, false>(r, local % ng, local / ng, ctl);
				return;
			}
		}
		if constexpr (MODE != 1)
			rho_body<D, 8, false, false>(r, local % ng, local / ng, ctl);
	} else if (phase == 1) {
		const ReduceArgs &r = stage_desc(A.red + b, item_desc().red);
		ctl.stage = MODE == 2 ? nullptr : r.stage;
		ctl.ready = A.count + b;
		ctl.ready_need = (unsigned)(__ldg(A.pre + b + 1) - __ldg(A.pre + b)) + (b == 0 ? A.phantom : 0u);
		reduce_body_wide(r, local, ctl);
	} else {
		const ForceArgs &f = stage_desc(A.force + b, item_desc().force);
		const int *stage = f.stage;
		const bool mixed = MODE == 1 || (MODE == 2 && stage && *(volatile const int *)stage == 0);
		ctl.stage = MODE == 2 ? nullptr : stage;
		ctl.ready = A.count + A.B + b;
		ctl.ready_need = (unsigned)(__ldg(A.pre + (A.B + 1) + b + 1) - __ldg(A.pre + (A.B + 1) + b));
		const int pg = __ldg(A.shape + 2 * A.B + b);
		if constexpr (MODE != 0) {
			if (mixed) {
				force_body<D, 8, true>(f, local % pg, local / pg, ctl);
				return;
			}
		}
		if constexpr (MODE != 1)
			force_body<D, 8, false>(f, local % pg, local / pg, ctl);
	}
}

// Queue position -> (phase, instance, item within the instance's phase): rho items first; then, instance by instance,
// its reduce items followed by its force items.
__device__ __forceinline__ int4 mbatch_decode(const MBatchArgs &A, int item)
{
	const int T0 = A.total[0];
	if (item < T0) {
		const int b = find_instance(A.pre, A.B, item);
		return make_int4(item, 0, b, item - __ldg(A.pre + b));
	}
	const int *prf = A.pre + 3 * (A.B + 1);
	const int li = item - T0;
	const int b = find_instance(prf, A.B, li);
	const int within = li - __ldg(prf + b);
	const int nred = __ldg(A.pre + (A.B + 1) + b + 1) - __ldg(A.pre + (A.B + 1) + b);
	return within < nred ? make_int4(item, 1, b, within) : make_int4(item, 2, b, within - nred);
}

template <int MODE>
__global__ void __launch_bounds__(kMBatchThreads, 3) cc_mbatch_kernel(MBatchArgs A)
{
	__shared__ int4 sh_item;   // the current item: (queue position, phase, instance, item within the phase)
	const int T = A.total[0] + A.total[1] + A.total[2];
	// Under programmatic dependent launch this grid may be scheduled while the previous one still takes items from
	// the same queue (its blocks trigger after their first item): wait for it to complete before taking any.
	cudaGridDependencySynchronize();
	for (;;) {
		__syncthreads();   // the previous item's shared memory is no longer read
		if (threadIdx.x == 0) {
			const int item = (int)atomicAdd(A.queue, 1u);
			sh_item = item < T ? mbatch_decode(A, item) : make_int4(item, 0, 0, 0);
		}
		__syncthreads();
		const int4 it = sh_item;
		if (it.x >= T)
			break;
		const int d = __ldg(A.dim + it.z);
		if (d == 3)
			mbatch_item<3, MODE>(A, it.y, it.z, it.w);
		else if (d == 2)
			mbatch_item<2, MODE>(A, it.y, it.z, it.w);
		else
			mbatch_item<1, MODE>(A, it.y, it.z, it.w);
		// the item's results are visible before its count rises
		__threadfence();
		__syncthreads();
		if (threadIdx.x == 0) {
			const int phase = it.y, b = it.z;
			const int *pre = A.pre + phase * (A.B + 1);
			unsigned *cnt = A.count + phase * A.B + b;
			const unsigned done = atomicAdd(cnt, 1u) + 1u;
			if (phase == 2 && done == (unsigned)(__ldg(pre + b + 1) - __ldg(pre + b))) {
				// the instance's last item: its counts start from zero in the next launch
				A.count[b] = 0u;
				A.count[A.B + b] = 0u;
				*cnt = 0u;
			}
		}
	}
	queue_leave(A.queue);
}

// ---------------------------------------------------------------------------------------------------------------
// Monte Carlo trial move: one particle from s_prev to s_after (ShiftedCCPotential_ForMC::TryMove)
// ---------------------------------------------------------------------------------------------------------------
// rho'(k) = rho(k) - exp(i k.r_prev) + exp(i k.r_after); dE = sum_k V (|rho'|^2 - |rho|^2) / Volume, with the change
// formed as 2 Re(conj(rho) delta) + |delta|^2 (no cancellation between two whole energies). Block partial sums in a
// fixed order; cc_mc_sum_kernel adds the blocks in order.
constexpr int kMcThreads = 256;

static __global__ void __launch_bounds__(kMcThreads) cc_mc_kernel(const int32_t *__restrict__ modes, int D,
                                                                  const double *__restrict__ V,
                                                                  const double2 *__restrict__ rho, int M, double sp0,
                                                                  double sp1, double sp2, double sa0, double sa1,
                                                                  double sa2, double2 *__restrict__ rho_trial,
                                                                  double *__restrict__ bpart)
{
	__shared__ double sh[kMcThreads / 32];
	const int m = blockIdx.x * kMcThreads + threadIdx.x;
	double e = 0.0;
	if (m < M) {
		const double sp[3] = {sp0, sp1, sp2}, sa[3] = {sa0, sa1, sa2};
		double hp = 0, lp = 0, ha = 0, la = 0;
		for (int c = 0; c < D; c++) {
			const int n = modes[(size_t)m * D + c];
			acc_phase(n, sp[c], hp, lp);
			acc_phase(n, sa[c], ha, la);
		}
		double tp = __dadd_rn(hp, lp), ta = __dadd_rn(ha, la);
		tp = __dsub_rn(tp, rint(tp));
		ta = __dsub_rn(ta, rint(ta));
		const double2 zp = expi2pi(tp), za = expi2pi(ta);
		const double2 r = rho[m];
		const double2 dl = make_double2(za.x - zp.x, za.y - zp.y);
		rho_trial[m] = make_double2(r.x + dl.x, r.y + dl.y);
		e = V[m] * (2.0 * (r.x * dl.x + r.y * dl.y) + dl.x * dl.x + dl.y * dl.y);
	}
	for (int o = 16; o > 0; o >>= 1)
		e += __shfl_down_sync(0xffffffffu, e, o);
	if ((threadIdx.x & 31) == 0)
		sh[threadIdx.x >> 5] = e;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < kMcThreads / 32; w++)
			t += sh[w];
		bpart[blockIdx.x] = t;
	}
}

static __global__ void cc_mc_sum_kernel(const double *__restrict__ bpart, int nb, double inv_vol, double *out,
                                        double shift = 0.0)
{
	double t = 0.0;
	for (int b = threadIdx.x; b < nb; b += 32)
		t += bpart[b];
	for (int o = 16; o > 0; o >>= 1)
		t += __shfl_down_sync(0xffffffffu, t, o);
	if (threadIdx.x == 0)
		*out = t * inv_vol + shift;
}

// ShiftedCCPotential_S2_MultiConfig (potential/CollectiveCoordinatePotential.h:1777-1870) over nsub sub-configurations
// whose rho per slot are rho[c * nslot + slot]: Snow = sum_c |rho_c|^2 / count (count = Np nsub), dS = Snow - S0,
// u_c = V dS conj(rho_c) for every c (the force pass of sub-configuration c reads u_c), and per-block partials of
// V dS^2 in bpart[blockIdx.x].
constexpr int kS2mThreads = 256;
static __global__ void __launch_bounds__(kS2mThreads)
cc_s2multi_kernel(const double2 *__restrict__ rho, double2 *__restrict__ u, int nslot, int nsub,
                  const double *__restrict__ slotV, const double *__restrict__ slotS0, double count,
                  double *__restrict__ bpart)
{
	__shared__ double sh[kS2mThreads / 32];
	const int slot = blockIdx.x * kS2mThreads + threadIdx.x;
	double e = 0.0;
	if (slot < nslot) {
		double snow = 0.0;
		for (int c = 0; c < nsub; c++) {
			const double2 r = rho[(size_t)c * nslot + slot];
			snow += r.x * r.x + r.y * r.y;
		}
		const double ds = snow / count - slotS0[slot];
		const double w = slotV[slot] * ds;
		e = w * ds;
		for (int c = 0; c < nsub; c++) {
			const double2 r = rho[(size_t)c * nslot + slot];
			u[(size_t)c * nslot + slot] = make_double2(w * r.x, -w * r.y);
		}
	}
	for (int o = 16; o > 0; o >>= 1)
		e += __shfl_down_sync(0xffffffffu, e, o);
	if ((threadIdx.x & 31) == 0)
		sh[threadIdx.x >> 5] = e;
	__syncthreads();
	if (threadIdx.x == 0) {
		double t = 0.0;
		for (int w = 0; w < kS2mThreads / 32; w++)
			t += sh[w];
		bpart[blockIdx.x] = t;
	}
}

}  // namespace cc
