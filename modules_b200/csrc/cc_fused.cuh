// cc_fused.cuh — one cooperative kernel per evaluation (small and medium problems).
//
// The three passes of cc_kernels.cuh become phases of one persistent grid (launched cooperatively, so every block is
// resident), separated by grid barriers:
//   phase 0  per-particle phase tables over the k-set's full index ranges, written once to global memory (L2) in two
//            layouts: particle-major (rho phase: a warp reads one particle's row) and entry-major (force phase: a
//            warp reads one entry of 32 consecutive particles);
//   phase 1  rho partials: work item = (group of 32 segments, particle split); one segment per lane, the 8 warps
//            stride over the split's particles; warps are summed in warp order into one partial row per split;
//   phase 2  per slot: sum of the split rows in split order, rho, u = V conj(rho), the slot's energy term; each block
//            sums its slots' terms in a fixed order;
//   phase 3  forces: work item = (32 particles, segment split) as in cc_force_kernel; the splits of a particle group
//            are summed in split order by the last item to finish (atomic ticket, no wait). Block 0 sums the blocks'
//            energy terms in block order.
// Grid barrier: every block's thread 0 takes an arrival ticket; the last arrival releases the others by bumping a
// generation word. The wait is bounded (kBarrierSpins polls with nanosleep); a block whose wait runs out sets the error
// word and every block leaves at its next barrier, so a fault in the barrier ends the launch instead of hanging it.
#pragma once
#include "cc_kernels.cuh"

namespace cc {

struct FusedArgs {
	const double *frac;       // N x D
	int N;
	// k-set
	const Seg *segs;          // ngroups * 32
	int ngroups, nseg, nslot; // nseg = ngroups * 32, nslot = nseg * L
	const double *slotV;
	double rho_offset, inv_vol, shift;
	// global tables
	TabSpec spec;             // one spec for every segment
	void *tabP;               // [N][rowP] particle-major (rowP = spec.row | 1)
	void *tabE;               // [row][Npad] entry-major (Npad = N rounded up to 32)
	int Npad;
	// rho
	int nsplit, per_split;
	double2 *partial;         // [nsplit][nslot]
	double2 *rho_slot, *u_slot;
	double *eblock;           // [gridDim.x]
	// force
	const int *kstart;        // nksplit + 1
	int nksplit;
	double *partialG;         // [nksplit][N][D] when nksplit > 1
	unsigned *fcounters;      // [ceil(N/32)]
	double recip[9];
	double fscale;
	double *F_out, *gfrac_out, *E_out;
	// barrier
	unsigned *bar;            // [0] arrivals, [1] generation, [2] error word
};

constexpr int kFusedThreads = 256;
constexpr int kFusedWarps = 8;
constexpr unsigned kBarrierSpins = 1u << 22;

// returns false when a barrier of this launch has failed (every thread of the block gets the same answer)
__device__ __forceinline__ bool grid_barrier(unsigned *bar)
{
	__shared__ int ok;
	__syncthreads();
	if (threadIdx.x == 0) {
		volatile unsigned *vgen = bar + 1;
		volatile unsigned *verr = bar + 2;
		const unsigned gen = *vgen;
		__threadfence();
		if (atomicAdd(bar, 1u) == gridDim.x - 1) {
			bar[0] = 0u;
			__threadfence();
			atomicAdd(bar + 1, 1u);
		} else {
			unsigned it = 0;
			while (*vgen == gen && *verr == 0u) {
				if (++it > kBarrierSpins) {
					atomicExch(bar + 2, 1u);
					break;
				}
				__nanosleep(64);
			}
		}
		__threadfence();
		ok = (*verr == 0u);
	}
	__syncthreads();
	return ok != 0;
}

template <int D, int L, bool MIXED>
__global__ void __launch_bounds__(kFusedThreads, 2) cc_fused_kernel(FusedArgs a)
{
	typedef typename std::conditional<MIXED, float, double>::type R;
	typedef typename std::conditional<MIXED, float2, double2>::type C;
	__shared__ double2 red[kFusedWarps * L * 32];   // phase 1: [warp][r][lane]
	__shared__ double sh_g[kFusedWarps * 32 * D];   // phase 3
	__shared__ double sh_e[kFusedWarps];
	__shared__ int sh_last;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const TabSpec &sp = a.spec;
	const int rowP = sp.row | 1;
	C *tabP = reinterpret_cast<C *>(a.tabP);
	C *tabE = reinterpret_cast<C *>(a.tabE);

	// ---- phase 0: tables -------------------------------------------------------------------------------------
	{
		const int total = a.N * sp.items;
		for (int t = blockIdx.x * kFusedThreads + threadIdx.x; t < total; t += gridDim.x * kFusedThreads) {
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
			const double s = a.frac[(size_t)j * D + run.axis];
			const int k0 = k * 8;
			double2 z = expi2pi(phase1(run.m0 + run.stride * k0, s));
			const double2 step = expi2pi(phase1(run.stride, s));
			const int k1 = min(run.count, k0 + 8);
			for (int kk = k0; kk < k1; kk++) {
				const C v = to_c<C>(z);
				tabP[(size_t)j * rowP + run.off + kk] = v;
				tabE[(size_t)(run.off + kk) * a.Npad + j] = v;
				z = cmul(z, step);
			}
		}
	}
	if (!grid_barrier(a.bar))
		return;

	// ---- phase 1: rho partials -------------------------------------------------------------------------------
	{
		const int items = a.ngroups * a.nsplit;
		for (int it = blockIdx.x; it < items; it += gridDim.x) {
			const int group = it % a.ngroups, split = it / a.ngroups;
			const Seg sg = a.segs[group * 32 + lane];
			SeedIdx ix = seed_index<D>(sp, sg);
			if (sg.len == 0) {
#pragma unroll
				for (int e = 0; e < 3; e++) {
					ix.a[e] = 0;
					ix.b[e] = -1;
				}
			}
			const int j0 = min(a.N, split * a.per_split), j1 = min(a.N, j0 + a.per_split);
			double2 acc[L];
#pragma unroll
			for (int r = 0; r < L; r++)
				acc[r] = make_double2(0.0, 0.0);
			int j = j0 + warp;
			for (; j + kFusedWarps < j1; j += 2 * kFusedWarps) {
				const C *r0 = tabP + (size_t)j * rowP, *r1 = r0 + (size_t)kFusedWarps * rowP;
				C z0 = seed_from_l2<D, C>(r0, 1, ix), z1 = seed_from_l2<D, C>(r1, 1, ix);
				const C w0 = __ldcg(r0 + ix.w), w1 = __ldcg(r1 + ix.w);
#pragma unroll
				for (int r = 0; r < L; r++) {
					acc[r].x += (double)(z0.x + z1.x);
					acc[r].y += (double)(z0.y + z1.y);
					z0 = cmul(z0, w0);
					z1 = cmul(z1, w1);
				}
			}
			if (j < j1) {
				const C *r0 = tabP + (size_t)j * rowP;
				C z0 = seed_from_l2<D, C>(r0, 1, ix);
				const C w0 = __ldcg(r0 + ix.w);
#pragma unroll
				for (int r = 0; r < L; r++) {
					acc[r].x += (double)z0.x;
					acc[r].y += (double)z0.y;
					z0 = cmul(z0, w0);
				}
			}
#pragma unroll
			for (int r = 0; r < L; r++)
				red[(warp * L + r) * 32 + lane] = acc[r];
			__syncthreads();
			for (int q = threadIdx.x; q < 32 * L; q += kFusedThreads) {   // q = r * 32 + lane
				double2 t = red[q];
				for (int w = 1; w < kFusedWarps; w++) {
					t.x += red[w * 32 * L + q].x;
					t.y += red[w * 32 * L + q].y;
				}
				a.partial[(size_t)split * a.nslot + (size_t)(q >> 5) * a.nseg + group * 32 + (q & 31)] = t;
			}
			__syncthreads();
		}
	}
	if (!grid_barrier(a.bar))
		return;

	// ---- phase 2: split sums, rho, u, energy terms ------------------------------------------------------------
	{
		double e = 0.0;
		for (int slot = blockIdx.x * kFusedThreads + threadIdx.x; slot < a.nslot; slot += gridDim.x * kFusedThreads) {
			double2 t = make_double2(0.0, 0.0);
			int sp2 = 0;
			for (; sp2 + 4 <= a.nsplit; sp2 += 4) {
				const double2 v0 = __ldcg(&a.partial[(size_t)sp2 * a.nslot + slot]);
				const double2 v1 = __ldcg(&a.partial[(size_t)(sp2 + 1) * a.nslot + slot]);
				const double2 v2 = __ldcg(&a.partial[(size_t)(sp2 + 2) * a.nslot + slot]);
				const double2 v3 = __ldcg(&a.partial[(size_t)(sp2 + 3) * a.nslot + slot]);
				t.x += v0.x;
				t.y += v0.y;
				t.x += v1.x;
				t.y += v1.y;
				t.x += v2.x;
				t.y += v2.y;
				t.x += v3.x;
				t.y += v3.y;
			}
			for (; sp2 < a.nsplit; sp2++) {
				const double2 v = __ldcg(&a.partial[(size_t)sp2 * a.nslot + slot]);
				t.x += v.x;
				t.y += v.y;
			}
			t.x += a.rho_offset;
			a.rho_slot[slot] = t;
			const double v = a.slotV[slot];
			a.u_slot[slot] = make_double2(v * t.x, -v * t.y);
			e += v * (t.x * t.x + t.y * t.y);
		}
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
			e += __shfl_down_sync(0xffffffffu, e, o);
		if (lane == 0)
			sh_e[warp] = e;
		__syncthreads();
		if (threadIdx.x == 0) {
			double b = 0.0;
			for (int w = 0; w < kFusedWarps; w++)
				b += sh_e[w];
			a.eblock[blockIdx.x] = b;
		}
	}
	if (!grid_barrier(a.bar))
		return;

	// ---- phase 3: forces --------------------------------------------------------------------------------------
	if (blockIdx.x == 0 && warp == 0) {
		double e = 0.0;
		for (int b = lane; b < (int)gridDim.x; b += 32)
			e += __ldcg(&a.eblock[b]);
#pragma unroll
		for (int o = 16; o > 0; o >>= 1)
			e += __shfl_down_sync(0xffffffffu, e, o);
		if (lane == 0)
			*a.E_out = e * a.inv_vol + a.shift;
	}
	if (a.F_out == nullptr && a.gfrac_out == nullptr)
		return;
	const int pgroups = (a.N + 31) / 32;
	const int fitems = pgroups * a.nksplit;
	for (int it = blockIdx.x; it < fitems; it += gridDim.x) {
		const int pg = it % pgroups, ks = it / pgroups;
		const int j = pg * 32 + lane;
		const int jj = min(j, a.N - 1);
		const int q0 = a.kstart[ks], q1 = a.kstart[ks + 1];
		double g[D];
#pragma unroll
		for (int e = 0; e < D; e++)
			g[e] = 0.0;
		const C *col = tabE + jj;
		for (int q = q0 + warp; q < q1; q += kFusedWarps) {
			const Seg sgm = a.segs[q];
			if (sgm.len == 0)
				continue;
			const SeedIdx ix = seed_index<D>(sp, sgm);
			C z = seed_from_l2<D, C>(col, (size_t)a.Npad, ix);
			const C w = __ldcg(col + (size_t)ix.w * a.Npad);
			const double2 *uq = a.u_slot + q;
			R S0 = 0, S1 = 0;
#pragma unroll
			for (int r = 0; r < L; r++) {
				const C uu = to_c<C>(__ldcg(uq + (size_t)r * a.nseg));
				const R t = uu.x * z.y + uu.y * z.x;
				S0 += t;
				S1 = fma((R)r, t, S1);
				z = cmul(z, w);
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
			if (a.nksplit == 1) {
				if (j < a.N)
					write_force_out<D>(a.F_out, a.gfrac_out, a.recip, a.fscale, j, t);
			} else {
				if (j < a.N) {
#pragma unroll
					for (int e = 0; e < D; e++)
						a.partialG[((size_t)ks * a.N + j) * D + e] = t[e];
				}
				__threadfence();
				__syncwarp();
				if (lane == 0)
					sh_last = (atomicAdd(&a.fcounters[pg], 1u) == (unsigned)(a.nksplit - 1));
				__syncwarp();
				if (sh_last) {
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
						write_force_out<D>(a.F_out, a.gfrac_out, a.recip, a.fscale, j, v);
					}
					if (lane == 0)
						a.fcounters[pg] = 0u;
				}
			}
		}
		__syncthreads();
	}
}

}  // namespace cc
