// cc_lbfgs.cuh — device-resident limited-memory BFGS for the collective-coordinate energy.
//
// Method: L-BFGS (Nocedal 1980) in the compact representation of Byrd, Nocedal and Schnabel (1994): with the m most
// recent pairs S = [s_i], Y = [y_i] (oldest first), R = upper triangle of S^T Y, D = diag(s_i^T y_i) and
// gamma = s^T y / y^T y of the newest pair,
//     H g = gamma g + S w1 + gamma Y w2,   t = R^-1 (S^T g),  w2 = -t,  w1 = R^-T ((D + gamma Y^T Y) t - gamma Y^T g),
// which needs two passes over the history per iteration (the dot products S^T g, Y^T g, ... and the combination),
// both parallel over the n = N d variables, instead of the 2m dependent dot products of the two-loop recursion.
// Line search: Armijo backtracking (c1 = 1e-4) with a safeguarded quadratic step; a pair enters the history only if
// s^T y > 0. Variables are the fractional coordinates; the gradient is dPhi/ds from the force kernel.
//
// One iteration on the device (every instance of a batch at once, blockIdx.y = instance):
//   evaluation at x_trial -> E_t, g_t;  lb_dots: block partials of the dot products;
//   lb_solve (one block per instance): totals in block order, accept / reject, history matrices and R^-1 (kept
//     with the history: a column per new pair), the products of the compact form, the next step length and the stop
//     tests;  lb_update: history insert, x, g, the new direction and x_trial.
// Every sum has a fixed order, so a run repeats bitwise.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cc {

constexpr int kLbMaxHist = 64;
// Restarts of a stalled FP64 minimisation (line search without decrease, or relative change below ftol) while the
// energy is above the stop value: the history is dropped and the run continues from the last accepted point, up to
// this many times (the reference's driver restarts its optimiser in each of its three passes,
// potential/StructureOptimization.cpp:1046-1072; near chi = 1/2 some configurations need more).
constexpr int kLbRestarts = 8;
constexpr int kLbThreads = 256;

enum LbStatus {
	kLbRunning = 0,
	kLbStopval = 1,    // energy at or below the stop value
	kLbGtol = 2,       // max |g| at or below gtol
	kLbMaxEval = 3,    // evaluation limit
	kLbLineSearch = 4, // line search found no decrease
	kLbFtol = 5        // relative energy change below ftol on 3 consecutive accepted steps
};

struct LbState {
	// energies and step
	double E, Et, alpha, gd, gamma;
	double stopval, gtol, ftol;
	int64_t max_evals, evals, iters;
	int m, count, head;     // history size, pairs stored, ring slot of the oldest pair
	int status, accepted, rejects, small_steps;
	int restarts;           // fresh-history restarts after a stall short of the stop value (at most kLbRestarts)
	int newslot;            // ring slot the update kernel fills with the accepted pair, or -1
	int stage;              // precision stage of the evaluations: 0 mixed, 1 FP64
	int sched;              // 1: mixed precision until switch_E (or a stall), then FP64
	double switch_E;
	double gmax;            // max |g| at x
	double gg;              // g.g at x
	double w[2 * kLbMaxHist];
	double SY[kLbMaxHist * kLbMaxHist];   // SY[i * m + j] = s_i . y_j (ring slots)
	double YY[kLbMaxHist * kLbMaxHist];   // YY[i * m + j] = y_i . y_j
	double Ri[kLbMaxHist * kLbMaxHist];   // R^-1 by ring slots (upper triangle in chronological order)
	double Sg[kLbMaxHist], Yg[kLbMaxHist];// S^T g, Y^T g at x (ring slots)
};

// What the host reads of each instance between blocks of iterations (gathered into one array: one copy per check)
struct LbBrief {
	int64_t evals, iters;
	double E;
	int status, stage;
};

struct LbInst {
	int n;                  // variables
	int m;                  // history size (the state's m, here as well so that kernels know it one load earlier)
	double *x, *g, *d, *xt, *gt;
	double *S, *Y;          // [m][n] ring
	double *part;           // [nblk][kLbDots]
	LbState *st;
};

// dot products per block. For each used ring slot i: s_i.gt, y_i.gt, s_i.y', y_i.y', y_i.s' with the candidate pair
// s' = xt - x, y' = gt - g; then gt.d, gt.gt, s'.y', y'.y', y'.gt, max|gt|. Differences are formed before the
// products, so s'.y' and the history cross terms carry no cancellation.
__host__ __device__ constexpr int lb_ndots(int m) { return 5 * m + 6; }

// Blocks of the dot-product kernel for an instance of n variables: one variable per thread (kLbThreads per block),
// at most `cap` blocks. A function of n and the cap only, so an instance's sums do not depend on the rest of a batch.
__host__ __device__ constexpr int lb_blocks(int n, int cap)
{
	return n <= 0 ? 1 : ((n + kLbThreads - 1) / kLbThreads < cap ? (n + kLbThreads - 1) / kLbThreads : cap);
}
constexpr int kLbMaxBlocks = 64;   // cap of the batched minimisation and the server

// Block partials of the dot products. The block's variables are taken in chunks of kLbThreads: the chunk's g_t,
// y = g_t - g and s = x_t - x go to shared memory once; warp w then forms the five products of history pairs w, w + 8,
// w + 16, ... over the chunk (every lane up to 8 variables, loads issued together), so the pairs' loads run in
// parallel across warps instead of one pair after another. Sums have a fixed order (lanes by a fixed tree, chunks in
// order, warps in order for the non-pair products), so a run repeats bitwise.
constexpr int kLbDotsThreads = 2 * kLbThreads;   // a chunk of kLbThreads variables; twice as many warps over the pairs
static __global__ void __launch_bounds__(kLbDotsThreads) lb_dots_kernel(const LbInst *insts, int cap, LbInst one)
{
	cudaGridDependencySynchronize();   // launched early (programmatic dependent launch): the evaluation is complete
	const LbInst in = insts ? insts[blockIdx.y] : one;
	const LbState *st = in.st;
	const int nblk = lb_blocks(in.n, cap);
	if ((int)blockIdx.x >= nblk)
		return;
	constexpr int kWarps = kLbDotsThreads / 32;
	const int m = in.m, nd = lb_ndots(m);
	const int per = (in.n + nblk - 1) / nblk;
	const int j0 = blockIdx.x * per, j1 = min(in.n, j0 + per);
	__shared__ double sgt[kLbThreads], syn[kLbThreads], ssn[kLbThreads];
	__shared__ double pr[5 * kLbMaxHist];
	__shared__ double red[kWarps][6];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	// the state's words and the first chunk's values go out together (the values' addresses do not depend on them)
	const int status = st->status, count = st->count;
	double v_gt = 0.0, v_g = 0.0, v_xt = 0.0, v_x = 0.0, v_d = 0.0;
	if (threadIdx.x < min(kLbThreads, j1 - j0)) {
		const int j = j0 + threadIdx.x;
		v_gt = in.gt[j];
		v_g = in.g[j];
		v_xt = in.xt[j];
		v_x = in.x[j];
		v_d = in.d[j];
	}
	if (status != kLbRunning)
		return;
	double a[6] = {0, 0, 0, 0, 0, 0};
	for (int k = threadIdx.x; k < 5 * count; k += kLbDotsThreads)
		pr[k] = 0.0;
	for (int c0 = j0; c0 < j1; c0 += kLbThreads) {
		const int cn = min(kLbThreads, j1 - c0);
		__syncthreads();   // the previous chunk is no longer read
		if (threadIdx.x < cn) {
			const int j = c0 + threadIdx.x;
			if (c0 != j0) {
				v_gt = in.gt[j];
				v_g = in.g[j];
				v_xt = in.xt[j];
				v_x = in.x[j];
				v_d = in.d[j];
			}
			const double gt = v_gt, yj = gt - v_g, sj = v_xt - v_x;
			a[0] += gt * v_d;
			a[1] += gt * gt;
			a[2] += sj * yj;
			a[3] += yj * yj;
			a[4] += yj * gt;
			a[5] = fmax(a[5], fabs(gt));
			sgt[threadIdx.x] = gt;
			syn[threadIdx.x] = yj;
			ssn[threadIdx.x] = sj;
		}
		__syncthreads();
		// two history pairs per step (i and i + kWarps): both pairs' loads are in flight together
		for (int i = warp; i < count; i += 2 * kWarps) {
			const int i2 = i + kWarps;
			const bool two = i2 < count;
			const double *s = in.S + (size_t)i * in.n + c0, *y = in.Y + (size_t)i * in.n + c0;
			const double *s2 = in.S + (size_t)(two ? i2 : i) * in.n + c0, *y2 = in.Y + (size_t)(two ? i2 : i) * in.n + c0;
			double si[kLbThreads / 32], yi[kLbThreads / 32], si2[kLbThreads / 32], yi2[kLbThreads / 32];
#pragma unroll
			for (int e = 0; e < kLbThreads / 32; e++) {
				const int k = lane + 32 * e;
				si[e] = k < cn ? s[k] : 0.0;
				yi[e] = k < cn ? y[k] : 0.0;
				si2[e] = k < cn && two ? s2[k] : 0.0;
				yi2[e] = k < cn && two ? y2[k] : 0.0;
			}
			double b[5] = {0, 0, 0, 0, 0}, b2[5] = {0, 0, 0, 0, 0};
#pragma unroll
			for (int e = 0; e < kLbThreads / 32; e++) {
				const int k = lane + 32 * e;
				if (k < cn) {
					b[0] += si[e] * sgt[k];
					b[1] += yi[e] * sgt[k];
					b[2] += si[e] * syn[k];
					b[3] += yi[e] * syn[k];
					b[4] += yi[e] * ssn[k];
					b2[0] += si2[e] * sgt[k];
					b2[1] += yi2[e] * sgt[k];
					b2[2] += si2[e] * syn[k];
					b2[3] += yi2[e] * syn[k];
					b2[4] += yi2[e] * ssn[k];
				}
			}
#pragma unroll
			for (int k = 0; k < 5; k++)
				for (int o = 16; o > 0; o >>= 1) {
					b[k] += __shfl_down_sync(0xffffffffu, b[k], o);
					b2[k] += __shfl_down_sync(0xffffffffu, b2[k], o);
				}
			if (lane == 0) {
				for (int k = 0; k < 5; k++)
					pr[5 * i + k] += b[k];
				if (two)
					for (int k = 0; k < 5; k++)
						pr[5 * i2 + k] += b2[k];
			}
		}
	}
#pragma unroll
	for (int k = 0; k < 5; k++)
		for (int o = 16; o > 0; o >>= 1)
			a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
	for (int o = 16; o > 0; o >>= 1)
		a[5] = fmax(a[5], __shfl_down_sync(0xffffffffu, a[5], o));
	if (lane == 0)
		for (int k = 0; k < 6; k++)
			red[warp][k] = a[k];
	__syncthreads();
	double *out = in.part + (size_t)blockIdx.x * nd;
	for (int k = threadIdx.x; k < nd; k += kLbDotsThreads) {
		if (k < 5 * m) {
			out[k] = k / 5 < count ? pr[k] : 0.0;
			continue;
		}
		const int q = k - 5 * m;
		double t = red[0][q];
		for (int w = 1; w < kWarps; w++)
			t = (q == 5) ? fmax(t, red[w][q]) : t + red[w][q];
		out[k] = t;
	}
}


// warp-wide sum with a fixed tree (every lane gets the total)
__device__ __forceinline__ double lb_warp_sum(double v)
{
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

constexpr int kLbSolveThreads = 256;

// Dynamic shared memory of lb_solve_kernel: the ring copies of S^T Y, Y^T Y and R^-1.
constexpr size_t kLbSolveSmem = 3 * sizeof(double) * kLbMaxHist * kLbMaxHist;

// One block per instance: block totals of the dot products (parallel over the products, blocks summed in order),
// accept / reject and the step length (thread 0), history matrices (parallel over slots), the products with R^-1 of
// the compact form, g.d of the new direction and the stop tests. R^-1 is kept with the history instead of solving
// with R each iteration: dropping the oldest pair keeps the trailing block of the inverse of an upper triangular
// matrix, and a new (newest) pair adds one column, -R^-1 r / rho with r_a = s_a . y_new and rho = s_new . y_new; so
// both triangular solves become matrix-vector products spread over the warps, where substitution was a chain of k
// dependent steps. The kernel is a chain of dependent phases, so its global reads are issued together up front: the
// partial sums, the state's scalars (thread 0) and the history matrices, which the block keeps in shared memory and
// updates there as well.
static __global__ void __launch_bounds__(kLbSolveThreads, 2) lb_solve_kernel(const LbInst *insts, int cap, LbInst one)
{
	cudaGridDependencySynchronize();
	const LbInst in = insts ? insts[blockIdx.x] : one;
	LbState *st = in.st;
	const int nblk = lb_blocks(in.n, cap);
	extern __shared__ double lb_smem[];
	double *shSY = lb_smem;                             // S^T Y by ring slots, m x m
	double *shYY = shSY + kLbMaxHist * kLbMaxHist;      // Y^T Y by ring slots, m x m
	double *shRi = shYY + kLbMaxHist * kLbMaxHist;      // R^-1 by ring slots, m x m
	__shared__ double tot[5 * kLbMaxHist + 6];
	__shared__ double Sg[kLbMaxHist], Yg[kLbMaxHist], t[kLbMaxHist], q[kLbMaxHist], w1[kLbMaxHist];
	__shared__ int slot[kLbMaxHist];
	__shared__ int sh_accept;
	const int status0 = st->status, m = in.m, nd = lb_ndots(m);
	const int count = st->count;
	// the state's scalars (loaded with the status word, and in flight while the partial sums load): every thread
	// takes the acceptance test and the new pair's slot, thread 0 the rest of the bookkeeping
	const double alpha = st->alpha, E = st->E, Et = st->Et, gd = st->gd, gamma0 = st->gamma;
	const int head = st->head;
	double stopval = 0.0, gtol = 0.0, ftol = 0.0, switch_E = 0.0;
	int64_t evals = 0, max_evals = 0, iters = 0;
	int rejects = 0, small = 0, restarts = 0, stage = 0, sched = 0;
	if (threadIdx.x == 0) {
		stopval = st->stopval;
		gtol = st->gtol;
		ftol = st->ftol;
		switch_E = st->switch_E;
		evals = st->evals;
		max_evals = st->max_evals;
		iters = st->iters;
		rejects = st->rejects;
		small = st->small_steps;
		restarts = st->restarts;
		stage = st->stage;
		sched = st->sched;
	}
	// The history matrices and the partial sums are loaded before the status word is tested: their addresses do not
	// depend on it, so all of these loads are in flight together (a finished instance loads them for nothing).
	// (eight elements of each matrix per thread in flight: a rolled loop would wait for each load before its store)
	for (int e0 = threadIdx.x; e0 < m * m; e0 += 8 * kLbSolveThreads) {
		double a[8], b[8], c[8];
#pragma unroll
		for (int u = 0; u < 8; u++) {
			const int e = e0 + u * kLbSolveThreads;
			a[u] = e < m * m ? st->SY[e] : 0.0;
			b[u] = e < m * m ? st->YY[e] : 0.0;
			c[u] = e < m * m ? st->Ri[e] : 0.0;
		}
#pragma unroll
		for (int u = 0; u < 8; u++) {
			const int e = e0 + u * kLbSolveThreads;
			if (e < m * m) {
				shSY[e] = a[u];
				shYY[e] = b[u];
				shRi[e] = c[u];
			}
		}
	}
	// totals: the blocks' partials in block order, up to 16 blocks' loads in flight
	for (int p = threadIdx.x; p < nd; p += kLbSolveThreads) {
		const bool is_max = p == nd - 1;
		double v = in.part[p];
		for (int b0 = 1; b0 < nblk; b0 += 16) {
			double pv[16];
#pragma unroll
			for (int u = 0; u < 16; u++)
				pv[u] = b0 + u < nblk ? in.part[(size_t)(b0 + u) * nd + p] : 0.0;
#pragma unroll
			for (int u = 0; u < 16; u++)
				if (b0 + u < nblk)
					v = is_max ? fmax(v, pv[u]) : v + pv[u];
		}
		tot[p] = v;
	}
	if (status0 != kLbRunning)
		return;
	__syncthreads();
	const double gtd = tot[5 * m], gtgt = tot[5 * m + 1], sy = tot[5 * m + 2], yy = tot[5 * m + 3],
	             ygt = tot[5 * m + 4], gtmax = tot[5 * m + 5];
	const bool finite = isfinite(Et) && isfinite(gtgt);
	const bool armijo = finite && Et <= E + 1e-4 * alpha * gd;
	if (!armijo) {
		if (threadIdx.x == 0) {
			evals++;
			int status = kLbRunning;
			// backtrack: safeguarded quadratic model of the energy along d
			double a2 = 0.5 * alpha;
			if (finite) {
				const double den = 2.0 * (Et - E - gd * alpha);
				if (den > 0)
					a2 = -gd * alpha * alpha / den;
				a2 = fmin(fmax(a2, 0.1 * alpha), 0.5 * alpha);
			}
			rejects++;
			if (rejects > 60 || a2 < 1e-300)
				status = kLbLineSearch;
			else if (evals >= max_evals)
				status = kLbMaxEval;
			const bool mixed_stage = sched && stage == 0;
			st->evals = evals;
			st->accepted = 0;
			if (status == kLbLineSearch && (mixed_stage || (E > stopval && restarts < kLbRestarts))) {
				// the mixed stage stalled at its noise floor: continue in FP64 from x with a fresh history; an FP64
				// run that stalled short of the stop value: restart from x with a fresh history
				if (mixed_stage)
					st->stage = 1;
				else
					st->restarts = restarts + 1;
				st->status = kLbRunning;
				st->count = 0;
				st->head = 0;
				st->E = INFINITY;
				st->alpha = 0.0;
				st->rejects = 0;
				st->small_steps = 0;
			} else {
				st->alpha = a2;
				st->rejects = rejects;
				st->status = status;
			}
		}
		return;
	}
	// accepted: the new pair enters the history if s.y > 0
	const bool keep = sy > 1e-300 && yy > 0 && isfinite(sy) && isfinite(yy);
	int newslot = -1, k = count, head1 = head;
	double gamma = gamma0;
	if (keep) {
		newslot = count < m ? (head + count) % m : head;
		if (count < m)
			k = count + 1;
		else
			head1 = (head + 1) % m;
		gamma = sy / yy;
	}
	if (threadIdx.x == 0) {
		int status = kLbRunning, acc = 1;
		evals++;
		iters++;
		const double dE = E - Et;
		small = (isfinite(E) && dE <= ftol * fabs(E)) ? small + 1 : 0;
		if (Et <= stopval && !(sched && stage == 0))
			status = kLbStopval;
		else if (gtmax <= gtol)
			status = kLbGtol;
		else if (small >= 3)
			status = kLbFtol;
		else if (evals >= max_evals)
			status = kLbMaxEval;
		if (sched && stage == 0 && (Et <= switch_E || status == kLbGtol || status == kLbFtol)) {
			// switch to FP64: the accepted point is re-evaluated in FP64 as a fresh start (E = inf accepts it)
			status = kLbRunning;
			stage = 1;
			small = 0;
			acc = 2;
		} else if (status == kLbFtol && Et > stopval && restarts < kLbRestarts) {
			// stalled short of the stop value: restart from the accepted point with a fresh history
			status = kLbRunning;
			restarts++;
			small = 0;
			acc = 2;
		}
		st->evals = evals;
		st->accepted = 1;
		st->rejects = 0;
		st->iters = iters;
		st->small_steps = small;
		st->count = k;
		st->head = head1;
		st->gamma = gamma;
		st->newslot = newslot;
		st->E = Et;
		st->gmax = gtmax;
		st->gg = gtgt;
		st->status = status;
		st->stage = stage;
		st->restarts = restarts;
		sh_accept = acc;   // read after the barriers below
	}
	// history products at the new point (ring slots), the new pair's rows and columns of S^T Y and Y^T Y (in the
	// state and in the block's copies)
	for (int i = threadIdx.x; i < count; i += kLbSolveThreads) {
		if (i == newslot)   // the oldest pair, replaced by the new one below
			continue;
		Sg[i] = tot[5 * i];
		Yg[i] = tot[5 * i + 1];
		if (newslot >= 0) {
			const double a = tot[5 * i + 2], b = tot[5 * i + 4], c = tot[5 * i + 3];
			st->SY[i * m + newslot] = a;
			st->SY[newslot * m + i] = b;
			st->YY[i * m + newslot] = c;
			st->YY[newslot * m + i] = c;
			shSY[i * m + newslot] = a;
			shSY[newslot * m + i] = b;
			shYY[i * m + newslot] = c;
			shYY[newslot * m + i] = c;
		}
	}
	if (threadIdx.x == 0 && newslot >= 0) {
		st->SY[newslot * m + newslot] = sy;
		st->YY[newslot * m + newslot] = yy;
		shSY[newslot * m + newslot] = sy;
		shYY[newslot * m + newslot] = yy;
		Sg[newslot] = alpha * gtd;   // s'.gt with s' = alpha d (alpha of this accepted step)
		Yg[newslot] = ygt;
	}
	__syncthreads();
	const double gam = k > 0 ? gamma : 1.0;
	for (int i = threadIdx.x; i < k; i += kLbSolveThreads) {
		st->Sg[i] = Sg[i];
		st->Yg[i] = Yg[i];
		slot[i] = head1 + i < m ? head1 + i : head1 + i - m;   // chronological index -> ring slot
	}
	__syncthreads();
	// compact form (chronological index a <-> ring slot slot[a]). Every product with a k x k matrix runs on the whole
	// block at once: four lanes per row (64 rows, kLbMaxHist), each taking every fourth term in order, then a fixed
	// two-step tree (the four lanes of a row are adjacent lanes of one warp; rows beyond k add nothing)
	static_assert(kLbSolveThreads == 4 * kLbMaxHist, "four lanes per history row");
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int row = threadIdx.x >> 2, sub = threadIdx.x & 3;
	auto row_sum = [](double v) {
		v += __shfl_xor_sync(0xffffffffu, v, 1);
		return v + __shfl_xor_sync(0xffffffffu, v, 2);
	};
	if (newslot >= 0) {
		// the new pair's column of R^-1 (the new pair is the newest, chronological index k - 1)
		double v = 0.0;
		if (row < k - 1) {
			const int ia = slot[row];
			for (int b = row + sub; b < k - 1; b += 4)
				v += shRi[ia * m + slot[b]] * shSY[slot[b] * m + newslot];
		}
		v = row_sum(v);
		if (row < k - 1 && sub == 0) {
			const double c = -v / sy;
			shRi[slot[row] * m + newslot] = c;
			st->Ri[slot[row] * m + newslot] = c;
		}
		if (threadIdx.x == 0) {
			const double c = 1.0 / sy;
			shRi[newslot * m + newslot] = c;
			st->Ri[newslot * m + newslot] = c;
		}
		__syncthreads();
	}
	// t = R^-1 S^T g
	{
		double v = 0.0;
		if (row < k) {
			const int ia = slot[row];
			for (int b = row + sub; b < k; b += 4)
				v += shRi[ia * m + slot[b]] * Sg[slot[b]];
		}
		v = row_sum(v);
		if (row < k && sub == 0)
			t[row] = v;
	}
	__syncthreads();
	// q = D t + gamma Y^T Y t - gamma Y^T g
	{
		double v = 0.0;
		if (row < k) {
			const int ia = slot[row];
			for (int b = sub; b < k; b += 4)
				v += shYY[ia * m + slot[b]] * t[b];
		}
		v = row_sum(v);
		if (row < k && sub == 0) {
			const int ia = slot[row];
			q[row] = shSY[ia * m + ia] * t[row] + gam * v - gam * Yg[ia];
		}
	}
	__syncthreads();
	// w1 = R^-T q
	{
		double v = 0.0;
		if (row < k) {
			const int ib = slot[row];
			for (int a = sub; a <= row; a += 4)
				v += shRi[slot[a] * m + ib] * q[a];
		}
		v = row_sum(v);
		if (row < k && sub == 0)
			w1[row] = v;
	}
	__syncthreads();
	if (warp == 0) {
		// store per ring slot: w[slot] = w1, w[kLbMaxHist + slot] = -gamma t; g.d of d = -(gamma g + S w1 + gamma Y w2)
		double gdn = 0.0;
		for (int a = lane; a < k; a += 32) {
			const int ia = slot[a];
			st->w[ia] = w1[a];
			st->w[kLbMaxHist + ia] = -gam * t[a];
			gdn += w1[a] * Sg[ia] - gam * t[a] * Yg[ia];
		}
		gdn = lb_warp_sum(gdn);
		if (lane == 0 && sh_accept == 2) {
			// fresh start (stage switch, or a restart after a stall): move to the accepted point (the update kernel
			// does), drop the history, zero step
			st->count = 0;
			st->head = 0;
			st->newslot = -1;
			st->E = INFINITY;
			st->gamma = 1.0;
			st->gd = 0.0;
			st->alpha = 0.0;
		} else if (lane == 0) {
			gdn = -(gam * gtgt + gdn);
			int kk = k;
			st->gamma = gam;
			if (!(gdn < 0) || !isfinite(gdn)) {
				// not a descent direction: drop the history (and the pair just formed), restart from steepest descent
				gdn = -gtgt;
				st->count = 0;
				st->head = 0;
				st->gamma = 1.0;
				st->newslot = -1;
				kk = 0;
			}
			st->gd = gdn;
			// first step of a fresh history: at most 1e-2 of a cell per coordinate; afterwards the unit step
			st->alpha = (kk == 0) ? fmin(1.0, 1e-2 / fmax(gtmax, 1e-300)) : 1.0;
		}
	}
}

// accept: insert the pair, move x and g; then d = -(gamma g + S w1 + gamma Y w2) and x_trial = x + alpha d.
// reject: x_trial = x + alpha d. The history sum is taken in quarters of the pairs: quarter q's terms in order (the
// first quarter starting from gamma g), then (P0 + P1) + (P2 + P3). LANES = 4 gives each quarter its own lane (all
// of a lane's pairs loaded at once, the tree through two shuffles: the single-instance launch, whose time is latency);
// LANES = 1 takes the four quarters on one thread (the multi-instance launches, which have parallelism to spare). Both
// do the same arithmetic, so an instance's result does not depend on the launch it runs in. The state's scalars and
// the variable's values are loaded up front (the stores below may alias them as far as the compiler knows, which
// would otherwise order every load after them).
constexpr int kLbUpdPairs = kLbMaxHist / 4;   // pairs per quarter at most
// quarter q of the history sum on one lane, all of its pairs' loads at once
__device__ __forceinline__ double lb_quarter(const double *__restrict__ S, const double *__restrict__ Y,
                                             const double *__restrict__ w, size_t n, int head, int m, int count,
                                             int q, double v)
{
	const int per = (count + 3) / 4, c0 = q * per;
	double sv[kLbUpdPairs], yv[kLbUpdPairs], ws[kLbUpdPairs], wy[kLbUpdPairs];
#pragma unroll
	for (int u = 0; u < kLbUpdPairs; u++) {
		const int c = c0 + u;
		const bool on = u < per && c < count;
		const int i = !on ? 0 : head + c < m ? head + c : head + c - m;
		sv[u] = on ? S[i * n] : 0.0;
		yv[u] = on ? Y[i * n] : 0.0;
		ws[u] = on ? w[i] : 0.0;
		wy[u] = on ? w[kLbMaxHist + i] : 0.0;
	}
#pragma unroll
	for (int u = 0; u < kLbUpdPairs; u++)
		if (u < per && c0 + u < count)
			v = fma(wy[u], yv[u], fma(ws[u], sv[u], v));
	return v;
}
template <int LANES>
static __global__ void __launch_bounds__(kLbThreads, LANES == 1 ? 4 : 2)
    lb_update_kernel(const LbInst *insts, LbInst one)
{
	cudaGridDependencySynchronize();
	const LbInst in = insts ? insts[blockIdx.y] : one;
	const LbState *st = in.st;
	const int status = st->status, accepted = st->accepted;
	if (status != kLbRunning && !(accepted && status != kLbLineSearch))
		return;   // (the whole block: one instance)
	const int sub = threadIdx.x & (LANES - 1);
	const int j = blockIdx.x * (kLbThreads / LANES) + threadIdx.x / LANES;
	const bool mine = j < in.n && sub == 0;   // the lane that stores the variable's results
	if (LANES == 1 && j >= in.n)
		return;
	const int jj = j < in.n ? j : 0;          // lanes past the end read variable 0 and store nothing
	const int m = st->m, newslot = st->newslot, count = st->count, head = st->head;
	const double gamma = st->gamma, alpha = st->alpha;
	const double xj = in.x[jj], xtj = in.xt[jj], gt = in.gt[jj], gj = in.g[jj];
	if (accepted) {
		if (mine) {
			if (newslot >= 0 && status == kLbRunning) {
				// s = x_trial - x exactly as stepped; y = gt - g (a finished run stores no pair, so a repeated
				// launch after the end only repeats the idempotent x = x_trial, g = gt)
				in.S[(size_t)newslot * in.n + j] = xtj - xj;
				in.Y[(size_t)newslot * in.n + j] = gt - gj;
			}
			in.x[j] = xtj;
			in.g[j] = gt;
		}
		if (status != kLbRunning)
			return;
		const double *S = in.S + jj, *Y = in.Y + jj, *w = st->w;
		const size_t n = (size_t)in.n;
		double v;
		if constexpr (LANES == 4) {
			v = lb_quarter(S, Y, w, n, head, m, count, sub, sub == 0 ? gamma * gt : 0.0);
			v += __shfl_xor_sync(0xffffffffu, v, 1);
			v += __shfl_xor_sync(0xffffffffu, v, 2);
		} else {
			// the same four quarter sums, one after another, each in batches of four pairs' loads
			const int per = (count + 3) / 4;
			double p[4];
#pragma unroll 1
			for (int q = 0; q < 4; q++) {
				double a = q == 0 ? gamma * gt : 0.0;
				const int c1 = min(count, (q + 1) * per);
				int c = q * per;
				for (; c + 4 <= c1; c += 4) {
					double sv[4], yv[4], ws[4], wy[4];
#pragma unroll
					for (int u = 0; u < 4; u++) {
						const int i = head + c + u < m ? head + c + u : head + c + u - m;
						sv[u] = S[i * n];
						yv[u] = Y[i * n];
						ws[u] = w[i];
						wy[u] = w[kLbMaxHist + i];
					}
#pragma unroll
					for (int u = 0; u < 4; u++)
						a = fma(wy[u], yv[u], fma(ws[u], sv[u], a));
				}
				for (; c < c1; c++) {
					const int i = head + c < m ? head + c : head + c - m;
					a = fma(w[kLbMaxHist + i], Y[i * n], fma(w[i], S[i * n], a));
				}
				p[q] = a;
			}
			v = (p[0] + p[1]) + (p[2] + p[3]);
		}
		if (mine) {
			in.d[j] = -v;
			in.xt[j] = xtj + alpha * -v;
		}
		return;
	}
	if (mine)
		in.xt[j] = xj + alpha * in.d[j];
}

static __global__ void lb_brief_kernel(const LbInst *insts, int count, LbBrief *out)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < count) {
		const LbState *st = insts[i].st;
		out[i] = LbBrief{st->evals, st->iters, st->E, st->status, st->stage};
	}
}

// The three kernels of one L-BFGS step on stream st for `count` instances (insts), at most `cap` dot-product blocks
// per instance and `maxn` variables in the largest one. Each is launched with programmatic stream serialisation:
// it is scheduled while the previous kernel drains and waits for it (cudaGridDependencySynchronize) before it reads.
// With one instance and its descriptor on the host (`one`), the descriptor goes in the kernels' parameters instead
// of being read from device memory (one dependent load fewer at the start of each kernel).
static inline cudaError_t lb_step(const LbInst *insts, int count, int cap, int maxn, cudaStream_t st,
                                  const LbInst *one = nullptr)
{
	const LbInst o = one && count == 1 ? *one : LbInst{};
	if (one && count == 1)
		insts = nullptr;
	static const cudaError_t smem_attr = cudaFuncSetAttribute(
	    lb_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLbSolveSmem);
	if (smem_attr != cudaSuccess)
		return smem_attr;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = 1;
	cudaLaunchConfig_t cfg = {};
	cfg.stream = st;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	cfg.gridDim = dim3(cap, count);
	cfg.blockDim = dim3(kLbDotsThreads);
	cudaError_t e = cudaLaunchKernelEx(&cfg, lb_dots_kernel, insts, cap, o);
	if (e != cudaSuccess)
		return e;
	cfg.gridDim = dim3(count);
	cfg.blockDim = dim3(kLbSolveThreads);
	cfg.dynamicSmemBytes = kLbSolveSmem;
	if ((e = cudaLaunchKernelEx(&cfg, lb_solve_kernel, insts, cap, o)) != cudaSuccess)
		return e;
	cfg.blockDim = dim3(kLbThreads);
	cfg.dynamicSmemBytes = 0;
	if (count == 1) {
		cfg.gridDim = dim3((maxn + kLbThreads / 4 - 1) / (kLbThreads / 4), 1);
		return cudaLaunchKernelEx(&cfg, lb_update_kernel<4>, insts, o);
	}
	cfg.gridDim = dim3((maxn + kLbThreads - 1) / kLbThreads, count);
	return cudaLaunchKernelEx(&cfg, lb_update_kernel<1>, insts, o);
}

}  // namespace cc
