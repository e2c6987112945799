// cc_batch.cuh — one cooperative launch evaluates many independent configurations (a batch of instances of one
// dimension D, each with its own cell, constraint set and particle count).
//
// The phases of cc_fused.cuh run over the union of every instance's work items; an item's instance is found by a
// binary search in the phase's prefix sums of item counts, so uneven instances balance over the persistent grid:
//   phase 0  per-particle phase tables of every instance (global memory, particle- and entry-major);
//   phase 1  rho partials: (instance, group of 32 segments, particle split of kBatchSplit particles);
//   phase 2  (instance, 256 slots): split sums, rho, u = V conj(rho), the chunk's energy term;
//   phase 3  forces: (instance, 32 particles, segment split of kBatchSegs segments); the item (0, 0) of an instance
//            also sums its energy terms in chunk order. Splits of a particle group are summed in split order by the last
//            item to finish (atomic ticket, no wait).
// An instance whose status word is nonzero (a finished minimisation) is skipped item by item. Grid barriers as in
// cc_fused.cuh (bounded waits).
#pragma once
#include "cc_fused.cuh"

namespace cc {

constexpr int kBatchSplit = 64;   // particles per rho item
constexpr int kBatchSegs = 64;    // segments per force item

struct BInst {
	const double *frac;       // N x D
	double *E_out, *gfrac_out, *F_out;   // outputs (F_out / gfrac_out may be null)
	const int *status;        // skip the instance when *status != 0 (null: never)
	const int *stage;         // skip the instance when *stage differs from the launch's stage (null: never)
	int N, Npad;
	const Seg *segs;
	int ngroups, nseg, nslot;
	const double *slotV;
	double rho_offset, inv_vol, shift;
	TabSpec spec;
	void *tabP, *tabE;
	int nsplit;
	double2 *partial;         // [nsplit][nslot]
	double2 *u_slot;          // [nslot]
	double *epart;            // [nechunk]
	int nechunk;              // ceil(nslot / 256)
	int nks;                  // force splits
	double *partialG;         // [nks][N][D]
	unsigned *fcounters;      // [ceil(N/32)]
	double recip[9];
	double fscale;
};

struct BatchArgs {
	const BInst *inst;
	int B;
	const int *pre[4];        // per phase: B + 1 prefix sums of item counts
	unsigned *bar;
};

__device__ __forceinline__ int batch_find(const int *pre, int B, int item)
{
	int lo = 0, hi = B;   // pre[lo] <= item < pre[hi]
	while (hi - lo > 1) {
		const int mid = (lo + hi) >> 1;
		if (__ldg(pre + mid) <= item)
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

__device__ __forceinline__ bool batch_skip(const BInst &in, int launch_stage)
{
	return (in.status && *(volatile const int *)in.status) ||
	       (in.stage && *(volatile const int *)in.stage != launch_stage);
}

template <int D, int L, bool MIXED>
__global__ void __launch_bounds__(kFusedThreads, 2) cc_batch_kernel(BatchArgs a)
{
	typedef typename std::conditional<MIXED, float, double>::type R;
	typedef typename std::conditional<MIXED, float2, double2>::type C;
	__shared__ double2 red[kFusedWarps * L * 32];
	__shared__ double sh_g[kFusedWarps * 32 * D];
	__shared__ double sh_e[kFusedWarps];
	__shared__ int sh_last;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

	// ---- phase 0: tables (item = one block of 256 table work items of one instance) --------------------------
	{
		const int items = a.pre[0][a.B];
		for (int it = blockIdx.x; it < items; it += gridDim.x) {
			const int b = batch_find(a.pre[0], a.B, it);
			const BInst &in = a.inst[b];
			if (batch_skip(in, MIXED ? 0 : 1))
				continue;
			const TabSpec &sp = in.spec;
			const int rowP = sp.row | 1;
			C *tabP = reinterpret_cast<C *>(in.tabP);
			C *tabE = reinterpret_cast<C *>(in.tabE);
			const int t = (it - a.pre[0][b]) * kFusedThreads + threadIdx.x;
			if (t >= in.N * sp.items)
				continue;
			const int j = t / sp.items;
			int k = t - j * sp.items;
			int r = 0;
			int nb = (sp.run[0].count + 7) >> 3;
			while (k >= nb) {
				k -= nb;
				r++;
				nb = (sp.run[r].count + 7) >> 3;
			}
			const TabRun &run = sp.run[r];
			const double s = in.frac[(size_t)j * D + run.axis];
			const int k0 = k * 8;
			double2 z = expi2pi(phase1(run.m0 + run.stride * k0, s));
			const double2 step = expi2pi(phase1(run.stride, s));
			const int k1 = min(run.count, k0 + 8);
			for (int kk = k0; kk < k1; kk++) {
				const C v = to_c<C>(z);
				tabP[(size_t)j * rowP + run.off + kk] = v;
				tabE[(size_t)(run.off + kk) * in.Npad + j] = v;
				z = cmul(z, step);
			}
		}
	}
	if (!grid_barrier(a.bar))
		return;

	// ---- phase 1: rho partials -------------------------------------------------------------------------------
	{
		const int items = a.pre[1][a.B];
		for (int it = blockIdx.x; it < items; it += gridDim.x) {
			const int b = batch_find(a.pre[1], a.B, it);
			const BInst &in = a.inst[b];
			if (batch_skip(in, MIXED ? 0 : 1))
				continue;
			const int local = it - a.pre[1][b];
			const int group = local % in.ngroups, split = local / in.ngroups;
			const TabSpec &sp = in.spec;
			const int rowP = sp.row | 1;
			const C *tabP = reinterpret_cast<const C *>(in.tabP);
			const Seg sg = in.segs[group * 32 + lane];
			SeedIdx ix = seed_index<D>(sp, sg);
			if (sg.len == 0) {
#pragma unroll
				for (int e = 0; e < 3; e++) {
					ix.a[e] = 0;
					ix.b[e] = -1;
				}
			}
			const int j0 = min(in.N, split * kBatchSplit), j1 = min(in.N, j0 + kBatchSplit);
			double2 acc[L];
#pragma unroll
			for (int r = 0; r < L; r++)
				acc[r] = make_double2(0.0, 0.0);
			int j = j0 + warp;
			for (; j + kFusedWarps < j1; j += 2 * kFusedWarps) {
				const C *r0 = tabP + (size_t)j * rowP, *r1 = r0 + (size_t)kFusedWarps * rowP;
				C z0 = seed_from_l2<D, C>(r0, 1, ix), z1 = seed_from_l2<D, C>(r1, 1, ix);
				const C w0 = __ldcg(r0 + ix.w), w1 = __ldcg(r1 + ix.w);
				if constexpr (MIXED) {
#pragma unroll
					for (int r = 0; r < L; r++) {
						acc[r].x += (double)z0.x + (double)z1.x;
						acc[r].y += (double)z0.y + (double)z1.y;
						z0 = cmul(z0, w0);
						z1 = cmul(z1, w1);
					}
				} else {
					const double c0 = 2.0 * w0.x, c1 = 2.0 * w1.x;
					double2 p0 = z0, p1 = z1, q0 = cmul(z0, w0), q1 = cmul(z1, w1);
					acc[0].x += p0.x + p1.x;
					acc[0].y += p0.y + p1.y;
					acc[1].x += q0.x + q1.x;
					acc[1].y += q0.y + q1.y;
#pragma unroll
					for (int r = 2; r < L; r++) {
						const double2 n0 = cheb_next(c0, q0, p0), n1 = cheb_next(c1, q1, p1);
						acc[r].x += n0.x + n1.x;
						acc[r].y += n0.y + n1.y;
						p0 = q0;
						q0 = n0;
						p1 = q1;
						q1 = n1;
					}
				}
			}
			if (j < j1) {
				const C *r0 = tabP + (size_t)j * rowP;
				C z0 = seed_from_l2<D, C>(r0, 1, ix);
				const C w0 = __ldcg(r0 + ix.w);
				if constexpr (MIXED) {
#pragma unroll
					for (int r = 0; r < L; r++) {
						acc[r].x += (double)z0.x;
						acc[r].y += (double)z0.y;
						z0 = cmul(z0, w0);
					}
				} else {
					const double c0 = 2.0 * w0.x;
					double2 p0 = z0, q0 = cmul(z0, w0);
					acc[0].x += p0.x;
					acc[0].y += p0.y;
					acc[1].x += q0.x;
					acc[1].y += q0.y;
#pragma unroll
					for (int r = 2; r < L; r++) {
						const double2 n0 = cheb_next(c0, q0, p0);
						acc[r].x += n0.x;
						acc[r].y += n0.y;
						p0 = q0;
						q0 = n0;
					}
				}
			}
#pragma unroll
			for (int r = 0; r < L; r++)
				red[(warp * L + r) * 32 + lane] = acc[r];
			__syncthreads();
			for (int q = threadIdx.x; q < 32 * L; q += kFusedThreads) {
				double2 t = red[q];
				for (int w = 1; w < kFusedWarps; w++) {
					t.x += red[w * 32 * L + q].x;
					t.y += red[w * 32 * L + q].y;
				}
				in.partial[(size_t)split * in.nslot + (size_t)(q >> 5) * in.nseg + group * 32 + (q & 31)] = t;
			}
			__syncthreads();
		}
	}
	if (!grid_barrier(a.bar))
		return;

	// ---- phase 2: split sums, rho, u, energy terms (item = 256 slots of one instance) --------------------------
	{
		const int items = a.pre[2][a.B];
		for (int it = blockIdx.x; it < items; it += gridDim.x) {
			const int b = batch_find(a.pre[2], a.B, it);
			const BInst &in = a.inst[b];
			if (batch_skip(in, MIXED ? 0 : 1))
				continue;
			const int chunk = it - a.pre[2][b];
			const int slot = chunk * kFusedThreads + threadIdx.x;
			double e = 0.0;
			if (slot < in.nslot) {
				double2 t = make_double2(0.0, 0.0);
				for (int sp2 = 0; sp2 < in.nsplit; sp2++) {
					const double2 v = __ldcg(&in.partial[(size_t)sp2 * in.nslot + slot]);
					t.x += v.x;
					t.y += v.y;
				}
				t.x += in.rho_offset;
				const double v = in.slotV[slot];
				in.u_slot[slot] = make_double2(v * t.x, -v * t.y);
				e = v * (t.x * t.x + t.y * t.y);
			}
#pragma unroll
			for (int o = 16; o > 0; o >>= 1)
				e += __shfl_down_sync(0xffffffffu, e, o);
			if (lane == 0)
				sh_e[warp] = e;
			__syncthreads();
			if (threadIdx.x == 0) {
				double s2 = 0.0;
				for (int w = 0; w < kFusedWarps; w++)
					s2 += sh_e[w];
				in.epart[chunk] = s2;
			}
			__syncthreads();
		}
	}
	if (!grid_barrier(a.bar))
		return;

	// ---- phase 3: forces and the energies ---------------------------------------------------------------------
	{
		const int items = a.pre[3][a.B];
		for (int it = blockIdx.x; it < items; it += gridDim.x) {
			const int b = batch_find(a.pre[3], a.B, it);
			const BInst &in = a.inst[b];
			if (batch_skip(in, MIXED ? 0 : 1))
				continue;
			const int local = it - a.pre[3][b];
			const int pgroups = (in.N + 31) / 32;
			const int pg = local % pgroups, ks = local / pgroups;
			if (local == 0 && warp == 0) {
				double e = 0.0;
				for (int c = lane; c < in.nechunk; c += 32)
					e += __ldcg(&in.epart[c]);
#pragma unroll
				for (int o = 16; o > 0; o >>= 1)
					e += __shfl_down_sync(0xffffffffu, e, o);
				if (lane == 0)
					*in.E_out = e * in.inv_vol + in.shift;
			}
			if (!in.F_out && !in.gfrac_out)
				continue;
			const TabSpec &sp = in.spec;
			const C *tabE = reinterpret_cast<const C *>(in.tabE);
			const int j = pg * 32 + lane;
			const int jj = min(j, in.N - 1);
			const int q0 = (int)((int64_t)in.nseg * ks / in.nks), q1 = (int)((int64_t)in.nseg * (ks + 1) / in.nks);
			double g[D];
#pragma unroll
			for (int e = 0; e < D; e++)
				g[e] = 0.0;
			const C *col = tabE + jj;
			for (int q = q0 + warp; q < q1; q += kFusedWarps) {
				const Seg sgm = in.segs[q];
				if (sgm.len == 0)
					continue;
				const SeedIdx ix = seed_index<D>(sp, sgm);
				C z = seed_from_l2<D, C>(col, (size_t)in.Npad, ix);
				const C w = __ldcg(col + (size_t)ix.w * in.Npad);
				const double2 *uq = in.u_slot + q;
				R S0 = 0, S1 = 0;
				if constexpr (MIXED) {
#pragma unroll
					for (int r = 0; r < L; r++) {
						const C uu = to_c<C>(__ldcg(uq + (size_t)r * in.nseg));
						const R t = uu.x * z.y + uu.y * z.x;
						S0 += t;
						S1 = fma((R)r, t, S1);
						z = cmul(z, w);
					}
				} else {
					double2 uu[L];
#pragma unroll
					for (int r = 0; r < L; r++)
						uu[r] = __ldcg(uq + (size_t)r * in.nseg);
					const double c = 2.0 * w.x;
					double2 p = z, qz = cmul(z, w);
					S0 = uu[0].x * p.y + uu[0].y * p.x;
					{
						const double t = uu[1].x * qz.y + uu[1].y * qz.x;
						S0 += t;
						S1 = t;
					}
#pragma unroll
					for (int r = 2; r < L; r++) {
						const double2 n = cheb_next(c, qz, p);
						const double t = uu[r].x * n.y + uu[r].y * n.x;
						S0 += t;
						S1 = fma((double)r, t, S1);
						p = qz;
						qz = n;
					}
				}
				const double S0d = (double)S0;
				if (D >= 2)
					g[0] = fma(S0d, (double)sgm.p0, g[0]);
				if (D >= 3)
					g[1] = fma(S0d, (double)sgm.p1, g[1]);
				g[D - 1] = fma(S0d, (double)sgm.start, g[D - 1] + (double)S1);
			}
#pragma unroll
			for (int e = 0; e < D; e++)
				sh_g[(warp * 32 + lane) * D + e] = g[e];
			__syncthreads();
			if (warp == 0) {
				double t[D];
#pragma unroll
				for (int e = 0; e < D; e++) {
					t[e] = sh_g[lane * D + e];
					for (int w2 = 1; w2 < kFusedWarps; w2++)
						t[e] += sh_g[(w2 * 32 + lane) * D + e];
				}
				if (in.nks == 1) {
					if (j < in.N)
						write_force_out<D>(in.F_out, in.gfrac_out, in.recip, in.fscale, j, t);
				} else {
					if (j < in.N) {
#pragma unroll
						for (int e = 0; e < D; e++)
							in.partialG[((size_t)ks * in.N + j) * D + e] = t[e];
					}
					__threadfence();
					__syncwarp();
					if (lane == 0)
						sh_last = (atomicAdd(&in.fcounters[pg], 1u) == (unsigned)(in.nks - 1));
					__syncwarp();
					if (sh_last) {
						__threadfence();
						if (j < in.N) {
							double v[D];
#pragma unroll
							for (int e = 0; e < D; e++)
								v[e] = __ldcg(&in.partialG[(size_t)j * D + e]);
							for (int k2 = 1; k2 < in.nks; k2++)
#pragma unroll
								for (int e = 0; e < D; e++)
									v[e] += __ldcg(&in.partialG[((size_t)k2 * in.N + j) * D + e]);
							write_force_out<D>(in.F_out, in.gfrac_out, in.recip, in.fscale, j, v);
						}
						if (lane == 0)
							in.fcounters[pg] = 0u;
					}
				}
			}
			__syncthreads();
		}
	}
}

}  // namespace cc
