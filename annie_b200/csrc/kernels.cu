// NTT passes of the modular-squaring engine, sm_100a.
//
// Mathematics (reference: ocl/kernel.cl and src/transformGPU.h of galloty/annie):
// per transform prime p_k, a register is n = 2^ln values.  The forward
// transform is LN-1 radix-2 levels; the level with S polynomials maps each
// block of 2m = n/S coefficients mod (x^2m - c^2) to mod (x^m - c) and
// (x^m + c) with c = w[S + j] (j = block index, twiddle table in bit-reversed
// order, transformGPU.h:117-160).  The product of the resulting degree-1
// polynomials is taken mod (x^2 -+ w[n/4 + q/2]) (kernel.cl:230-256), and the
// inverse levels undo the forward ones.  The transform primes are below 2^30,
// so values stay lazily reduced ([0, 4p) forward, [0, 2p) inverse; see
// arith.cuh) and every butterfly is one Shoup product and three adds.  Only
// the exact coefficient values that the carry produces are visible outside,
// and they do not depend on the primes or the order of the butterflies.
//
// This file splits the n coefficients 2-D (row*R + col): the column pass owns
// the first LA levels (all H rows of 32 adjacent columns, all KP primes, in
// shared memory) and the row pass owns the last LB levels (one row of one
// prime per CTA, 16 coefficients per thread in registers).
#include <atomic>
#include <utility>

#include "kernels.h"

namespace ab
{

// Programmatic dependent launch: the row, mid and column passes are launched
// so that the next pass on the stream may be scheduled while the current one
// is still running.  Until griddep_wait() a pass reads only what no earlier
// pass of the stream writes (twiddles, its launch parameters, the per-slot
// control words uploaded before a graph launch) and writes only shared
// memory; griddep_wait() returns once the previous kernel of the stream has
// completed and its writes are visible.  The next pass is scheduled as the
// CTAs of the current one exit (AB_PDL_TRIGGER 0).  An explicit trigger right
// after griddep_wait (1) or before the final stores (2) lets the next pass
// hold SM resources while this one still runs; both measured slower on B200
// (33.2 M bits: 221.7 and 233.3 us per squaring against 210.1; without PDL
// 218.9).
#ifndef AB_PDL
#define AB_PDL 1
#endif
#ifndef AB_PDL_TRIGGER
#define AB_PDL_TRIGGER 0
#endif
__device__ __forceinline__ void griddep_wait()
{
#if AB_PDL
	asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
__device__ __forceinline__ void griddep_launch()
{
#if AB_PDL && AB_PDL_TRIGGER == 1
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}
__device__ __forceinline__ void griddep_launch_late()
{
#if AB_PDL && AB_PDL_TRIGGER == 2
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// ================================================================ row pass
// A CTA transforms one row (R = 2^(LB+1) words) of one prime: levels
// t = 0..LB-1 of the row touch bit LB-t of the in-row index.  Each thread
// holds 16 words; a stage applies S <= 4 levels to groups of 2^S words in
// registers, and stages exchange through shared memory.  The last stage owns
// bits 4..1; bit 0 (the two halves of a degree-1 polynomial) comes from the
// thread index, so the pointwise product pairs lane 2m with lane 2m+1.
// Stage loops are rolled (runtime bit positions) to keep the code small.
constexpr int RP_EPT = 16;

// Twiddles of the row pass: the forward levels read w; the inverse levels
// read the -w^-1 table wi (domain R) or, for domain Q (wi == null), the
// forward table at the mirrored position of the level: the level with s
// polynomials holds indices [s, 2s), and index i mirrors to 3s - 1 - i.
struct RowTw
{
	const uint2 * w;
	const uint2 * wi;
	u32 H;
};

template <int S, bool INV>
__device__ __forceinline__ void rp_radix(u32 (&v)[RP_EPT], u32 tid, u32 T, int b, int LB, const RowTw & tw,
	u32 Hr, u32 p, u32 p2)
{
	constexpr int G = RP_EPT >> S;
#pragma unroll
	for (int x = 0; x < G; ++x)
	{
		const u32 ohi = (tid + T * (u32)x) >> b;
#pragma unroll
		for (int ss = 0; ss < S; ++ss)
		{
			const int s = INV ? ss : (S - 1 - ss);
			const int t = LB - b - s;
			const u32 i0 = (Hr << t) + (ohi << (S - 1 - s));
#pragma unroll
			for (int jh = 0; jh < (1 << (S - 1 - s)); ++jh)
			{
				uint2 wv;
				if (!INV) wv = __ldg(tw.w + i0 + jh);
				else if (tw.wi != nullptr) wv = __ldg(tw.wi + i0 + jh);
				else wv = __ldg(tw.w + (3u * (tw.H << t) - 1u - (i0 + jh)));
#pragma unroll
				for (int gl = 0; gl < (1 << s); ++gl)
				{
					const int g = x * (1 << S) + (jh << (s + 1)) + gl;
					if (INV) inv_bf(v[g], v[g + (1 << s)], wv.x, wv.y, p, p2);
					else fwd_bf(v[g], v[g + (1 << s)], wv.x, wv.y, p, p2);
				}
			}
		}
	}
}

// Stage addressing: the 2^S words of a group are e0 + g 2^b.  In the padded
// shared layout they are pad(e0) + g D with D = 2^b + 2^(b-4) for b >= 5, and
// D = 2 for the last stage (b = 1, the group stays inside one 32-word block).
__device__ __forceinline__ u32 rp_pad(u32 e) { return e + ((e >> 5) << 1); }

__device__ __forceinline__ u32 rp_base(u32 tid, u32 T, int x, int S, int b)
{
	const u32 o = tid + T * (u32)x;
	return (o & ((1u << b) - 1)) | ((o >> b) << (b + S));
}
__device__ __forceinline__ u32 rp_step(int b) { return (b >= 5) ? (1u << b) + (1u << (b - 4)) : (1u << b); }

template <int S>
__device__ __forceinline__ void rp_load_smem(u32 (&v)[RP_EPT], const u32 * sm, u32 tid, u32 T, int b)
{
	const u32 D = rp_step(b);
#pragma unroll
	for (int x = 0; x < (RP_EPT >> S); ++x)
	{
		const u32 * a = sm + rp_pad(rp_base(tid, T, x, S, b));
#pragma unroll
		for (int g = 0; g < (1 << S); ++g) v[x * (1 << S) + g] = a[g * D];
	}
}

template <int S>
__device__ __forceinline__ void rp_store_smem(const u32 (&v)[RP_EPT], u32 * sm, u32 tid, u32 T, int b)
{
	const u32 D = rp_step(b);
#pragma unroll
	for (int x = 0; x < (RP_EPT >> S); ++x)
	{
		u32 * a = sm + rp_pad(rp_base(tid, T, x, S, b));
#pragma unroll
		for (int g = 0; g < (1 << S); ++g) a[g * D] = v[x * (1 << S) + g];
	}
}

template <int S>
__device__ __forceinline__ void rp_load_global(u32 (&v)[RP_EPT], const u32 * __restrict__ x, u32 tid, u32 T, int b)
{
#pragma unroll
	for (int xx = 0; xx < (RP_EPT >> S); ++xx)
	{
		const u32 * a = x + rp_base(tid, T, xx, S, b);
#pragma unroll
		for (int g = 0; g < (1 << S); ++g) v[xx * (1 << S) + g] = a[(u32)g << b];
	}
}

template <int S>
__device__ __forceinline__ void rp_store_global(const u32 (&v)[RP_EPT], u32 * __restrict__ x, u32 tid, u32 T, int b)
{
#pragma unroll
	for (int xx = 0; xx < (RP_EPT >> S); ++xx)
	{
		u32 * a = x + rp_base(tid, T, xx, S, b);
#pragma unroll
		for (int g = 0; g < (1 << S); ++g) a[(u32)g << b] = v[xx * (1 << S) + g];
	}
}

// Pointwise product of the degree-1 polynomials (x0, x1) mod (x^2 -+ c):
// lane 2m holds the x0 of the thread pair's 16 polynomials, lane 2m+1 the x1.
// Each lane computes 8 whole products (even lane: slots 0..7, odd: 8..15).
// Inputs: [0, 4p) from the forward levels, the other operand in [0, 2p);
// every product is a Montgomery product (a factor 2^-32 that the carry's CRT
// weights remove); outputs in [0, 2p) for the inverse levels.
// w1: the 8 twiddles of the thread pair's last forward level (just read by
// the forward stage, so an L1 hit), which are the polynomials' c.
__device__ __forceinline__ void rp_pointwise(u32 (&v)[RP_EPT], const u32 * __restrict__ xp, bool is_mul, u32 tid, u32 NT,
	const uint2 * __restrict__ w1, u32 p, u32 p2, u32 pinv)
{
	// tid: virtual thread (its 16 words are the last-stage elements
	// 32*(tid>>1) + (tid&1) + 2g); NT: physical threads of the CTA (warp mask)
	const bool odd = (tid & 1) != 0;
	const unsigned mask = (NT >= 32) ? 0xffffffffu : ((1u << NT) - 1);
	const u32 * __restrict__ xq = is_mul ? xp + (tid & 1) + ((tid >> 1) << 5) : nullptr;
#pragma unroll
	for (int i = 0; i < 8; ++i)
	{
		const u32 r = __shfl_xor_sync(mask, odd ? v[i] : v[8 + i], 1);
		const u32 x0 = red2(odd ? r : v[i], p2), x1 = red2(odd ? v[8 + i] : r, p2);
		const int slot = odd ? 8 + i : i;   // polynomial slot; parity = sign
		const uint2 cwp = __ldg(w1 + (odd ? 4 + (i >> 1) : (i >> 1)));
		const u32 cw = cwp.x, cs = cwp.y;
		u32 y0, y1, t;
		if (is_mul)
		{
			const u32 pa = __ldg(xq + 2 * i), pb = __ldg(xq + 2 * (8 + i));
			const u32 rp2 = __shfl_xor_sync(mask, odd ? pa : pb, 1);
			const u32 p0 = odd ? rp2 : pa, p1 = odd ? pb : rp2;
			t = shoup(mont(x1, p1, p, pinv), cw, cs, p);
			y1 = red2(mont(x0, p1, p, pinv) + mont(x1, p0, p, pinv), p2);
			y0 = mont(x0, p0, p, pinv);
		}
		else
		{
			t = shoup(mont(x1, x1, p, pinv), cw, cs, p);
			y1 = mont(red2(x0 + x0, p2), x1, p, pinv);
			y0 = mont(x0, x0, p, pinv);
		}
		y0 = red2(((slot & 1) == 0) ? y0 + t : y0 - t + p2, p2);
		const u32 r2 = __shfl_xor_sync(mask, odd ? y0 : y1, 1);
		if (odd) { v[8 + i] = y1; v[i] = r2; }
		else { v[i] = y0; v[8 + i] = r2; }
	}
}

template <int N>
__device__ __forceinline__ void reduce_all(u32 (&v)[N], u32 p2)
{
#pragma unroll
	for (int i = 0; i < N; ++i) v[i] = red2(v[i], p2);
}

// Physical threads of a row-pass CTA: 16 words per virtual thread, at most
// 256 threads, each running R / (16 * threads) rounds per stage.  The kernel
// is compiled for 4 CTAs per SM (at most 64 registers), so that the Q- and
// R-domain row passes, which run side by side on two streams, are resident
// together.
#ifndef AB_ROW_THREADS
#define AB_ROW_THREADS 256
#endif
#ifndef AB_ROW_MINB
#define AB_ROW_MINB 4
#endif
template <int LOG_R>
struct RowCfg
{
	static constexpr u32 T = (1u << LOG_R) / RP_EPT;             // virtual threads
	static constexpr u32 NT = (T < AB_ROW_THREADS) ? T : AB_ROW_THREADS;   // physical threads
	static constexpr u32 RND = T / NT;
	static constexpr int MINB = (AB_ROW_MINB * AB_ROW_THREADS > 2048) ? 2048 / AB_ROW_THREADS : AB_ROW_MINB;
	static constexpr size_t SMEM = sizeof(u32) * ((1u << LOG_R) + (1u << LOG_R) / 16);   // padded row
};

// The row pass of row bx (prime k = bx / HR, row r) of candidate cand, by P
// threads (tid < P) sharing the padded row buffer sm.  When P exceeds the
// row's virtual threads T, the threads above T only take part in the
// barriers.  mask_nt: threads of the CTA, for the shuffle masks.
template <int LOG_R, u32 P>
__device__ __forceinline__ void rowpass_body(const RowJob & J, const TConst & c, u32 cand, u32 bx, u32 tid, u32 * sm, u32 mask_nt)
{
	constexpr int LB = LOG_R - 1;
	constexpr u32 T = RowCfg<LOG_R>::T, NT = P, RND = (T + P - 1) / P;
	constexpr bool IDLE = P > T;                                  // some threads have no virtual thread
	constexpr int NL = LB - 4;                                    // levels above the last stage
	constexpr int S0 = (NL % 4 == 0) ? 4 : NL % 4;                // first stage (when NL > 0)
	constexpr int NS = (NL == 0) ? 0 : 1 + (NL - S0) / 4;        // stages above the last
	constexpr int B0 = LB + 1 - S0;

	const size_t cofs = (size_t)cand * J.stride;
	const u32 k = bx / c.HR, r = bx - k * c.HR;
	const u32 p = c.p[k], p2 = 2 * p, pinv = c.pinv[k];
	u32 * __restrict__ x = J.x + cofs + (size_t)k * c.n + (size_t)r * (1u << LOG_R);
	RowTw tw;
	tw.w = J.w + (size_t)k * (c.n >> 1);
	tw.wi = (J.wi != nullptr) ? J.wi + (size_t)k * (c.n >> 1) : nullptr;
	tw.H = c.HR;
	const u32 * __restrict__ xp = (J.mode == ROW_MUL) ? J.xp + cofs + (size_t)k * c.n + (size_t)r * (1u << LOG_R) : nullptr;
	const u32 Hr = c.HR + r;
	// threads of a shuffle: with idle threads, only the first T of the first warp
	const u32 mnt = (IDLE && T < 32) ? T : mask_nt;
	u32 v[RP_EPT];
	// twiddles of the last forward level of virtual thread vt: the c of its polynomials
	auto w1 = [&](u32 vt) { return tw.w + (Hr << (LB - 1)) + ((vt >> 1) << 3); };
	griddep_wait();
	griddep_launch();

	if constexpr (NS == 0)
	{
#pragma unroll 1
		for (u32 rr = 0; rr < RND; ++rr)
		{
			const u32 vt = tid + rr * NT;
			if (IDLE && vt >= T) continue;
			rp_load_global<4>(v, x, vt, T, 1);
			rp_radix<4, false>(v, vt, T, 1, LB, tw, Hr, p, p2);
			if (J.mode != ROW_FWD_ONLY)
			{
				rp_pointwise(v, xp, J.mode == ROW_MUL, vt, mnt, w1(vt), p, p2, pinv);
				rp_radix<4, true>(v, vt, T, 1, LB, tw, Hr, p, p2);
			}
			else reduce_all(v, p2);
			rp_store_global<4>(v, x, vt, T, 1);
		}
		return;
	}
	else
	{
		// ---- forward: stage 0 from global, then stages of 4 levels via smem
#pragma unroll 1
		for (u32 rr = 0; rr < RND; ++rr)
		{
			const u32 vt = tid + rr * NT;
			if (IDLE && vt >= T) continue;
			rp_load_global<S0>(v, x, vt, T, B0);
			rp_radix<S0, false>(v, vt, T, B0, LB, tw, Hr, p, p2);
			rp_store_smem<S0>(v, sm, vt, T, B0);
		}
		int b = B0;
#pragma unroll 1
		for (int i = 1; i < NS; ++i)
		{
			__syncthreads();
			b -= 4;
#pragma unroll 1
			for (u32 rr = 0; rr < RND; ++rr)
			{
				const u32 vt = tid + rr * NT;
			if (IDLE && vt >= T) continue;
				rp_load_smem<4>(v, sm, vt, T, b);
				rp_radix<4, false>(v, vt, T, b, LB, tw, Hr, p, p2);
				rp_store_smem<4>(v, sm, vt, T, b);
			}
		}
		__syncthreads();

		// ---- last stage (bits 4..1), pointwise, inverse last stage
#pragma unroll 1
		for (u32 rr = 0; rr < RND; ++rr)
		{
			const u32 vt = tid + rr * NT;
			if (IDLE && vt >= T) continue;
			rp_load_smem<4>(v, sm, vt, T, 1);
			rp_radix<4, false>(v, vt, T, 1, LB, tw, Hr, p, p2);
			if (J.mode == ROW_FWD_ONLY)
			{
				reduce_all(v, p2);
				rp_store_global<4>(v, x, vt, T, 1);
				continue;
			}
			rp_pointwise(v, xp, J.mode == ROW_MUL, vt, mnt, w1(vt), p, p2, pinv);
			rp_radix<4, true>(v, vt, T, 1, LB, tw, Hr, p, p2);
			rp_store_smem<4>(v, sm, vt, T, 1);
		}
		if (J.mode == ROW_FWD_ONLY) return;

		// ---- inverse: back up through smem, stage 0 to global
		b = 1;
#pragma unroll 1
		for (int i = NS - 1; i >= 1; --i)
		{
			__syncthreads();
			b += 4;
#pragma unroll 1
			for (u32 rr = 0; rr < RND; ++rr)
			{
				const u32 vt = tid + rr * NT;
			if (IDLE && vt >= T) continue;
				rp_load_smem<4>(v, sm, vt, T, b);
				rp_radix<4, true>(v, vt, T, b, LB, tw, Hr, p, p2);
				rp_store_smem<4>(v, sm, vt, T, b);
			}
		}
		__syncthreads();
		griddep_launch_late();
#pragma unroll 1
		for (u32 rr = 0; rr < RND; ++rr)
		{
			const u32 vt = tid + rr * NT;
			if (IDLE && vt >= T) continue;
			rp_load_smem<S0>(v, sm, vt, T, B0);
			rp_radix<S0, true>(v, vt, T, B0, LB, tw, Hr, p, p2);
			rp_store_global<S0>(v, x, vt, T, B0);
		}
	}
}

template <int LOG_R>
__global__ void __launch_bounds__(RowCfg<LOG_R>::NT, RowCfg<LOG_R>::MINB) k_rowpass(const RowJobs jobs, const TConst c)
{
	extern __shared__ __align__(16) u32 sm[];
	const RowJob J = (blockIdx.y == 0) ? jobs.j[0] : jobs.j[1];
	const u32 cand = blockIdx.z;
	if (J.active != nullptr && J.active[cand] == 0u) return;
	rowpass_body<LOG_R, RowCfg<LOG_R>::NT>(J, c, cand, blockIdx.x, threadIdx.x, sm, RowCfg<LOG_R>::NT);
}

// ================================================================ column pass
constexpr int CC = 32;  // own columns per CTA
#ifndef AB_COL_THREADS
#define AB_COL_THREADS 384
#endif
constexpr int COL_THREADS = AB_COL_THREADS;
constexpr int TW = 40;  // tile row stride: own columns + up to 8 predecessor columns

// One radix-2^S step of the column transform (levels on row bits b..b+S-1)
// for one column of one prime: the 2^S rows that differ in those bits.
// Global level l (2^l polynomials) works on row bit LOG_H-1-l with twiddle
// tw[2^l + j], j = row >> (LOG_H - l) (forward: w; inverse: -w^-1).
template <int S, bool INV>
__device__ __forceinline__ void col_step(u32 * __restrict__ colp, int LOG_H, int b, u32 o, const uint2 * __restrict__ tw,
	u32 p, u32 p2)
{
	u32 v[1 << S];
	const u32 row0 = (o & ((1u << b) - 1)) | ((o >> b) << (b + S));
	u32 * const base = colp + row0 * TW;
	const u32 D = (u32)TW << b;
#pragma unroll
	for (int g = 0; g < (1 << S); ++g) v[g] = base[g * D];
	const u32 ohi = o >> b;
#pragma unroll
	for (int ss = 0; ss < S; ++ss)
	{
		const int s = INV ? ss : (S - 1 - ss);
		const int lvl = LOG_H - 1 - (b + s);
		const uint2 * __restrict__ twl = tw + ((1u << lvl) + (ohi << (S - 1 - s)));
#pragma unroll
		for (int jh = 0; jh < (1 << (S - 1 - s)); ++jh)
		{
			const uint2 wv = twl[jh];
#pragma unroll
			for (int gl = 0; gl < (1 << s); ++gl)
			{
				const int g = (jh << (s + 1)) + gl;
				if (INV) inv_bf(v[g], v[g + (1 << s)], wv.x, wv.y, p, p2);
				else fwd_bf(v[g], v[g + (1 << s)], wv.x, wv.y, p, p2);
			}
		}
	}
#pragma unroll
	for (int g = 0; g < (1 << S); ++g) base[g * D] = v[g];
}

// One task of a column stage: column u of prime k, row group o.
template <int LOG_H, bool INV>
__device__ __forceinline__ void col_task(u32 * tile, int u, int o, int k, int S, int b, const uint2 * twk, const TConst & c)
{
	u32 * colp = tile + (k << LOG_H) * TW + u;
	const uint2 * tw = twk + (k << LOG_H);
	const u32 p = c.p[k];
	if (S == 3) col_step<3, INV>(colp, LOG_H, b, (u32)o, tw, p, 2 * p);
	else if (S == 2) col_step<2, INV>(colp, LOG_H, b, (u32)o, tw, p, 2 * p);
	else col_step<1, INV>(colp, LOG_H, b, (u32)o, tw, p, 2 * p);
}

// All LOG_H levels of the CC own columns [E, E + CC) and, with pred, the E
// predecessor columns [0, E) of every prime, in place in the tile; stages of
// 3 levels (the remainder first in the forward order).  Task indices split
// by shifts only (E is 0, 4 or 8).
template <int LOG_H, int KP, bool INV>
__device__ __forceinline__ void col_transform(u32 * tile, int E, bool pred, const uint2 * twk, const TConst & c)
{
	constexpr int SR = (LOG_H % 3 == 0) ? 3 : LOG_H % 3;       // top stage (row bits LOG_H-SR..LOG_H-1)
	constexpr int NST = 1 + (LOG_H - SR) / 3;
	static_assert(CC == 32, "32 own columns per CTA");
	const int tid = (int)threadIdx.x, NT = (int)blockDim.x;
	const int le = (E == 8) ? 3 : 2;                           // log2 E when E > 0
#pragma unroll 1
	for (int st = 0; st < NST; ++st)
	{
		// forward: top stage first; inverse: bottom stage first
		const int idx = INV ? (NST - 1 - st) : st;
		const bool top = (idx == 0);
		const int b = top ? (LOG_H - SR) : (LOG_H - SR - 3 * idx);
		const int S = top ? SR : 3;
		const int lo = LOG_H - S;                                // log2 of the row groups
		for (int task = tid; task < (KP << (lo + 5)); task += NT)
			col_task<LOG_H, INV>(tile, E + (task & 31), (task >> 5) & ((1 << lo) - 1), task >> (lo + 5), S, b, twk, c);
		if (pred && E > 0)
			for (int task = tid; task < (KP << (lo + le)); task += NT)
				col_task<LOG_H, INV>(tile, task & (E - 1), (task >> le) & ((1 << lo) - 1), task >> (lo + le), S, b, twk, c);
		__syncthreads();
	}
}

// Adds delta to the exact value of one coefficient (three limb planes, plane
// stride PS words).
__device__ __forceinline__ void exact_add(u32 * t, int PS, __int128 delta)
{
	const unsigned __int128 u = (unsigned __int128)t[0] | ((unsigned __int128)t[PS] << 32) | ((unsigned __int128)t[2 * PS] << 64);
	__int128 v = (__int128)(u << 32) >> 32;             // sign-extend the 96-bit value
	v += delta;
	const unsigned __int128 w = (unsigned __int128)v;
	t[0] = (u32)w; t[PS] = (u32)(w >> 32); t[2 * PS] = (u32)(w >> 64);
}

// Residues of the exact values of 4 coefficients (limb words l[0..2], each 4
// coefficients) in the KP planes of the tile at tp (plane stride PS words).
template <int KP>
__device__ __forceinline__ void encode4(const TConst & c, const uint4 (&l)[AB_NW], u32 * tp, int PS)
{
	const u32 d0[4] = { l[0].x, l[0].y, l[0].z, l[0].w };
	const u32 d1[4] = { l[1].x, l[1].y, l[1].z, l[1].w };
	const u32 d2[4] = { l[2].x ^ 0x80000000u, l[2].y ^ 0x80000000u, l[2].z ^ 0x80000000u, l[2].w ^ 0x80000000u };
#pragma unroll
	for (int k = 0; k < KP; ++k)
	{
		uint4 r;
		r.x = encode_res(c, k, d0[0], d1[0], d2[0]);
		r.y = encode_res(c, k, d0[1], d1[1], d2[1]);
		r.z = encode_res(c, k, d0[2], d1[2], d2[2]);
		r.w = encode_res(c, k, d0[3], d1[3], d2[3]);
		*reinterpret_cast<uint4 *>(tp + k * PS) = r;
	}
}

// Second carry phase for one group of 4 coefficients (kernel.cl:1582-1613):
// f = carry-in, d = the group's unsigned digits; returns each coefficient's
// exact value (balanced top digit, the last coefficient absorbing the rest)
// as three limbs and the top sub-digit of the last coefficient.
template <int L, int PCK>
__device__ __forceinline__ i32 carry_phase2(int lb, Big<L> f, const u32 (&d)[4][PCK], u32 (&x)[AB_NW][4])
{
	const i32 base = (i32)(1u << lb);
#pragma unroll
	for (int j = 0; j < 3; ++j)
	{
		f = add_digits<L, PCK>(f, lb, d[j]);
		u32 e[PCK];
		extract_shift<L, PCK>(f, lb, e);
		i32 top = (i32)e[PCK - 1];
		if (top >= base / 2) { top -= base; f = big_add_u32<L>(f, 1u); }
		digits_exact<PCK>(lb, top, e, x[0][j], x[1][j], x[2][j]);
	}
	f = add_digits<L, PCK>(f, lb, d[3]);
	const u32 bm = (u32)base - 1;
	u32 e[PCK];
	i32 top;
	if (PCK == 1)
	{
		top = (i32)(i64)big_low64<L>(f);
	}
	else if (PCK == 2)
	{
		const i64 r01 = (i64)big_low64<L>(f);
		e[0] = (u32)r01 & bm;
		top = (i32)(r01 >> lb);
	}
	else
	{
		const u64 r01 = big_low64<L>(f) & (((u64)1 << (2 * lb)) - 1);
		e[0] = (u32)r01 & bm;
		e[1 % PCK] = (u32)(r01 >> lb);
		const Big<L> f23 = big_sar<L>(f, 2 * lb);
		const i64 r23 = (i64)big_low64<L>(f23);
		e[2 % PCK] = (u32)r23 & bm;
		top = (i32)(r23 >> lb);
	}
	digits_exact<PCK>(lb, top, e, x[0][3], x[1][3], x[2][3]);
	return top;
}

// The column pass of column group b of nb (32 columns each) of candidate
// cand, by all threads of the CTA; sm: colpass_smem bytes of shared memory.
template <int LOG_H, int K, int PCK>
__device__ __forceinline__ void colpass_body(ColJob J, const TConst & c, u32 cand, int b, int nb, u32 * sm, int & decision)
{
	constexpr int KP = K + 1, L = K;             // transform primes, limbs of the carry
	constexpr int H = 1 << LOG_H;
	constexpr int PS = H * TW;                   // tile plane stride
	u32 * const tile = sm;                       // [KP][H][TW]
	u32 * const cw = tile + KP * PS;             // [H][TW/4][L] carry-out words
	uint2 * const twc = reinterpret_cast<uint2 *>(cw + H * (TW / 4) * L);   // [3][KP][H] column twiddles

	const u32 amul = (J.mult != nullptr) ? J.mult[cand] : J.a;
	if (amul == 0u) return;                       // inactive batch slot
	{
		const size_t on = (size_t)cand * J.stride_norm, ot = (size_t)cand * J.stride_ntt;
		J.in += J.transformed ? ot : on;
		if (J.sub) J.sub += on;
		if (J.out_norm) J.out_norm += on;
		if (J.out_fwd[0]) J.out_fwd[0] += ot;
		if (J.out_fwd[1]) J.out_fwd[1] += ot;
		if (J.out_snap) J.out_snap = (J.snap_flag[cand] != 0u) ? J.out_snap + on : nullptr;
	}
	const int lb = (J.cand != nullptr) ? J.cand[cand].lbase : c.lbase;
	const u32 R = c.R, n = c.n;
	const u32 c0 = (u32)b * CC;
	const bool single = (nb == 1);
	// predecessor columns: the 4 left of the CTA (the last 4 of the previous row
	// for CTA 0); CTA 0 also takes the 4 before those when the mod R / mod Q
	// decision needs the final top coefficient
	const int E = (!J.transformed || single) ? 0 : ((b == 0 && J.lower != LOWER_NONE) ? 8 : 4);
	const int WU = CC + E, ng = WU / 4;
	const int tid = (int)threadIdx.x, NT = (int)blockDim.x;

	auto gcol = [&](int u) -> u32 { return (u < E) ? ((b == 0) ? R - (u32)E + (u32)u : c0 - (u32)E + (u32)u) : c0 + (u32)(u - E); };

	// ---- the column twiddles (constant tables), then the tile (NTT form: KP
	// planes; normal form: the three limb planes), which the previous pass wrote
	for (int idx = tid; idx < KP * H; idx += NT)
	{
		const int k = idx / H, i = idx % H;
		if (i == 0) continue;
		if (J.transformed) twc[idx] = J.wi_in[k * COLTW + i];
		if (J.out_fwd[0] != nullptr) twc[KP * H + idx] = J.w_out[0][k * COLTW + i];
		if (J.out_fwd[1] != nullptr) twc[2 * KP * H + idx] = J.w_out[1][k * COLTW + i];
	}
	griddep_wait();
	griddep_launch();
	const int np_in = J.transformed ? KP : AB_NW;
	for (int idx = tid; idx < (np_in << (LOG_H + 3)); idx += NT)
	{
		const int u4 = idx & 7, row = (idx >> 3) & (H - 1), k = idx >> (LOG_H + 3);
		const uint4 val = __ldg(reinterpret_cast<const uint4 *>(J.in + (size_t)k * n + (size_t)row * R + c0 + 4 * u4));
		*reinterpret_cast<uint4 *>(tile + k * PS + row * TW + E + 4 * u4) = val;
	}
	if (E > 0)
	{
		const int le4 = (E == 8) ? 1 : 0;                          // log2 of the predecessor groups
		for (int idx = tid; idx < (np_in << (LOG_H + le4)); idx += NT)
		{
			const int u4 = idx & (E / 4 - 1), row = (idx >> le4) & (H - 1), k = idx >> (LOG_H + le4);
			const uint4 val = __ldg(reinterpret_cast<const uint4 *>(J.in + (size_t)k * n + (size_t)row * R + gcol(4 * u4)));
			*reinterpret_cast<uint4 *>(tile + k * PS + row * TW + 4 * u4) = val;
		}
	}
	if (tid == 0) decision = 0;
	__syncthreads();

	if (J.transformed)
	{
		// ---- inverse column levels (all WU columns, KP primes)
		col_transform<LOG_H, KP, true>(tile, E, true, twc, c);

		// ---- carry phase 1: per group, exact values (CRT), x a, - sub,
		// unsigned digits + carry-out
		const int npg = (E == 8) ? H + 1 : (E == 4) ? H : 0;    // predecessor groups carried (for E = 8 only row H-1's first)
		for (int idx = tid; idx < H * (CC / 4) + npg; idx += NT)
		{
			int row, u4;
			if (idx < H * (CC / 4)) { row = idx >> 3; u4 = E / 4 + (idx & 7); }
			else
			{
				const int q = idx - H * (CC / 4);
				if (E == 4) { row = q; u4 = 0; }
				else { row = (q < H) ? q : H - 1; u4 = (q < H) ? 1 : 0; }
			}
			u32 xv[KP][4];
#pragma unroll
			for (int k = 0; k < KP; ++k)
			{
				const uint4 t = *reinterpret_cast<const uint4 *>(tile + k * PS + row * TW + 4 * u4);
				xv[k][0] = t.x; xv[k][1] = t.y; xv[k][2] = t.z; xv[k][3] = t.w;
			}
			u32 sv[AB_NW][4];
			if (J.sub != nullptr)
			{
#pragma unroll
				for (int l = 0; l < AB_NW; ++l)
				{
					const uint4 t = __ldg(reinterpret_cast<const uint4 *>(J.sub + (size_t)l * n + (size_t)row * R + gcol(4 * u4)));
					sv[l][0] = t.x; sv[l][1] = t.y; sv[l][2] = t.z; sv[l][3] = t.w;
				}
			}
			Big<L> f = big_zero<L>();
			u32 dg[4][PCK];
#pragma unroll
			for (int j = 0; j < 4; ++j)
			{
				u32 rr[KP];
#pragma unroll
				for (int k = 0; k < KP; ++k) rr[k] = xv[k][j];
				Big<L> V = crt<L>(c, rr);
				if (amul != 1u) V = big_mul_u32<L>(V, amul);
				if (J.sub != nullptr) V = big_sub<L>(V, big_from_exact<L>(sv[0][j], sv[1][j], sv[2][j]));
				f = big_add<L>(f, V);
				extract_shift<L, PCK>(f, lb, dg[j]);
			}
#pragma unroll
			for (int l = 0; l < PCK; ++l)
				*reinterpret_cast<uint4 *>(tile + l * PS + row * TW + 4 * u4) = make_uint4(dg[0][l], dg[1][l], dg[2][l], dg[3][l]);
#pragma unroll
			for (int l = 0; l < L; ++l) cw[(row * (TW / 4) + u4) * L + l] = f.l[l];
		}
		__syncthreads();

		// ---- carry phase 2: add the previous group's carry-out, balanced
		// digits, exact values
		const int own_groups = CC / 4;
		for (int idx = tid; idx < H * own_groups + 1; idx += NT)
		{
			int row, u4;
			bool store = true;
			if (idx == H * own_groups)
			{
				// CTA 0 re-derives the last coefficient of the register from its
				// predecessor columns, for the mod R / mod Q decision
				if (E != 8) continue;
				row = H - 1; u4 = 1; store = false;
			}
			else
			{
				row = idx / own_groups; u4 = E / 4 + idx % own_groups;
			}
			int prow = row, pu4 = u4 - 1;
			bool neg = false;
			if (store && b == 0 && u4 == E / 4)
			{
				// first group of a row: its predecessor ends the previous row
				pu4 = (E == 0) ? (ng - 1) : (E / 4 - 1);
				if (row > 0) prow = row - 1;
				else { prow = H - 1; neg = (J.nega != 0); }
			}
			Big<L> f;
#pragma unroll
			for (int l = 0; l < L; ++l) f.l[l] = cw[(prow * (TW / 4) + pu4) * L + l];
			if (neg) f = big_neg<L>(f);
			u32 dg[4][PCK];
#pragma unroll
			for (int l = 0; l < PCK; ++l)
			{
				const uint4 t = *reinterpret_cast<const uint4 *>(tile + l * PS + row * TW + 4 * u4);
				dg[0][l] = t.x; dg[1][l] = t.y; dg[2][l] = t.z; dg[3][l] = t.w;
			}
			u32 ex[AB_NW][4];
			const i32 top = carry_phase2<L, PCK>(lb, f, dg, ex);
			if (store)
			{
#pragma unroll
				for (int l = 0; l < AB_NW; ++l)
					*reinterpret_cast<uint4 *>(tile + l * PS + row * TW + 4 * u4) = make_uint4(ex[l][0], ex[l][1], ex[l][2], ex[l][3]);
			}
			const bool is_last = (row == H - 1) && (u4 == ng - 1) && (b == nb - 1);
			if ((is_last || !store) && top >= (i32)(1u << lb)) decision = 1;
		}
		__syncthreads();

		// ---- mod R (+2) / mod Q on the top and bottom coefficients (kernel.cl:1653-1683)
		if (J.lower != LOWER_NONE && tid == 0)
		{
			if (decision && b == nb - 1) exact_add(tile + (H - 1) * TW + WU - 1, PS, -((__int128)1 << (c.pck * lb)));
			if (b == 0)
			{
				int d = 0;
				if (decision) d += (J.lower == LOWER_Q) ? -1 : 1;
				if (J.lower == LOWER_R_ADD2) d += 2;
				if (d != 0) exact_add(tile + E, PS, (__int128)d);
			}
		}
		__syncthreads();
	}

	griddep_launch_late();
	// ---- outputs: normal form, then the first LA forward levels of the next
	// product in one or two domains (the residues are encoded from the exact
	// values in the tile, or for the second domain from the normal form in
	// global memory)
	if (J.out_norm != nullptr || J.out_snap != nullptr)
	{
		for (int idx = tid; idx < AB_NW * H * (CC / 4); idx += NT)
		{
			const int u4 = idx % (CC / 4), row = (idx / (CC / 4)) % H, l = idx / ((CC / 4) * H);
			const uint4 val = *reinterpret_cast<const uint4 *>(tile + l * PS + row * TW + E + 4 * u4);
			const size_t o = (size_t)l * n + (size_t)row * R + c0 + 4 * u4;
			if (J.out_norm) *reinterpret_cast<uint4 *>(J.out_norm + o) = val;
			if (J.out_snap) *reinterpret_cast<uint4 *>(J.out_snap + o) = val;
		}
	}
	bool first = true;
#pragma unroll 1
	for (int dom = 0; dom < 2; ++dom)
	{
		u32 * const out = (dom == 0) ? J.out_fwd[0] : J.out_fwd[1];
		if (out == nullptr) continue;
		__syncthreads();
		const u32 * src = first ? nullptr : (J.transformed ? J.out_norm : J.in);
		for (int idx = tid; idx < H * (CC / 4); idx += NT)
		{
			const int u4 = idx % (CC / 4), row = idx / (CC / 4);
			u32 * const tp = tile + row * TW + E + 4 * u4;
			uint4 l[AB_NW];
#pragma unroll
			for (int i = 0; i < AB_NW; ++i)
				l[i] = (src == nullptr) ? *reinterpret_cast<const uint4 *>(tp + i * PS)
				                        : *reinterpret_cast<const uint4 *>(src + (size_t)i * n + (size_t)row * R + c0 + 4 * u4);
			encode4<KP>(c, l, tp, PS);
		}
		__syncthreads();
		col_transform<LOG_H, KP, false>(tile, E, false, twc + (1 + dom) * KP * H, c);
		for (int idx = tid; idx < KP * H * (CC / 4); idx += NT)
		{
			const int u4 = idx % (CC / 4), row = (idx / (CC / 4)) % H, k = idx / ((CC / 4) * H);
			*reinterpret_cast<uint4 *>(out + (size_t)k * n + (size_t)row * R + c0 + 4 * u4) =
				*reinterpret_cast<const uint4 *>(tile + k * PS + row * TW + E + 4 * u4);
		}
		first = false;
	}
}

template <int LOG_H, int K, int PCK>
__global__ void __launch_bounds__(COL_THREADS, 2) k_colpass(const ColJobs jobs, const TConst c)
{
	extern __shared__ __align__(16) u32 sm[];
	__shared__ int decision;
	colpass_body<LOG_H, K, PCK>((blockIdx.y == 0) ? jobs.j[0] : jobs.j[1], c, blockIdx.z, (int)blockIdx.x, (int)gridDim.x, sm, decision);
}

// ================================================================ mixed-size passes
// The class of CTA bid and the CTA's job, candidate and row / column group.
struct FusedCta
{
	int ci;
	u32 job, cand, bx;
};

template <typename Pass>
__device__ __forceinline__ FusedCta fused_cta(const Pass * __restrict__ d, u32 bid)
{
	FusedCta f;
	int ci = 0;
	while (ci + 1 < d->nclass && bid >= d->begin[ci + 1]) ++ci;
	const u32 local = bid - d->begin[ci], nbx = d->nbx[ci];
	const u32 cj = local / nbx;
	f.ci = ci;
	f.bx = local - cj * nbx;
	f.job = cj % d->njobs[ci];
	f.cand = cj / d->njobs[ci];
	return f;
}

// The class's constants into shared memory (they come from a table written
// when the group was set up, so before griddep_wait).
__device__ __forceinline__ void fused_consts(TConst & cs, const TConst * __restrict__ tcs, int ci)
{
	const u32 * src = reinterpret_cast<const u32 *>(tcs + ci);
	u32 * dst = reinterpret_cast<u32 *>(&cs);
	for (u32 i = threadIdx.x; i < sizeof(TConst) / 4; i += blockDim.x) dst[i] = __ldg(src + i);
	__syncthreads();
}

__global__ void __launch_bounds__(AB_FUSED_ROW_THREADS, 4) k_fused_rowpass(const FusedRowPass * __restrict__ d, const TConst * __restrict__ tcs)
{
	extern __shared__ __align__(16) u32 sm[];
	__shared__ TConst cs;
	const FusedCta f = fused_cta(d, blockIdx.x);
	const RowJob J = d->jobs[f.ci].j[f.job];
	if (J.active != nullptr && J.active[f.cand] == 0u) return;
	fused_consts(cs, tcs, f.ci);
	constexpr u32 P = AB_FUSED_ROW_THREADS;
	switch (d->log_r[f.ci])
	{
	case 5: rowpass_body<5, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 6: rowpass_body<6, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 7: rowpass_body<7, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 8: rowpass_body<8, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 9: rowpass_body<9, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 10: rowpass_body<10, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 11: rowpass_body<11, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 12: rowpass_body<12, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 13: rowpass_body<13, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	case 14: rowpass_body<14, P>(J, cs, f.cand, f.bx, threadIdx.x, sm, P); break;
	default: break;
	}
}

#define AB_FUSED_COL(LH, KK, PP) \
	case LH * 8 + KK: colpass_body<LH, KK, PP>(J, cs, f.cand, (int)f.bx, (int)d->nbx[f.ci], sm, decision); break;
#define AB_FUSED_COL_K(LH) AB_FUSED_COL(LH, 2, 1) AB_FUSED_COL(LH, 3, 2) AB_FUSED_COL(LH, 4, 2) AB_FUSED_COL(LH, 5, 4)

__global__ void __launch_bounds__(COL_THREADS, 2) k_fused_colpass(const FusedColPass * __restrict__ d, const TConst * __restrict__ tcs)
{
	extern __shared__ __align__(16) u32 sm[];
	__shared__ TConst cs;
	__shared__ int decision;
	const FusedCta f = fused_cta(d, blockIdx.x);
	const ColJob J = d->jobs[f.ci].j[f.job];
	const u32 amul = (J.mult != nullptr) ? J.mult[f.cand] : J.a;
	if (amul == 0u) return;                       // inactive batch slot
	fused_consts(cs, tcs, f.ci);
	switch (d->sel[f.ci])
	{
	AB_FUSED_COL_K(1) AB_FUSED_COL_K(2) AB_FUSED_COL_K(3) AB_FUSED_COL_K(4) AB_FUSED_COL_K(5) AB_FUSED_COL_K(6)
	default: break;
	}
}
#undef AB_FUSED_COL_K
#undef AB_FUSED_COL

// ================================================================ register words of the reference
// Canonical residue of the exact value (d0, d1, d2) mod a reference prime:
// d0 + d1 2^32 + d2 2^64 with Montgomery steps (r2 = 2^64 mod p, so
// ref_mont(x, r2) = x 2^32 mod p); a negative value is negated first.
__device__ __forceinline__ u32 ref_mont(u32 a, u32 b, u32 p, u32 q)
{
	const u64 t = (u64)a * b;
	const u32 m = (u32)t * q;
	return ref_sub((u32)(t >> 32), __umulhi(m, p), p);
}

__device__ __forceinline__ u32 ref_add(u32 a, u32 b, u32 p) { return ref_sub(a, p - b, p); }

__global__ void k_export(const RefConst rc, const u32 * __restrict__ norm, u32 * __restrict__ words, u32 n)
{
	const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	u32 d0 = norm[i], d1 = norm[n + i], d2 = norm[2 * (size_t)n + i];
	const bool neg = (i32)d2 < 0;
	if (neg)
	{
		// two's-complement negation of the 96-bit value
		d0 = ~d0; d1 = ~d1; d2 = ~d2;
		d0 += 1; if (d0 == 0) { d1 += 1; if (d1 == 0) d2 += 1; }
	}
	for (int k = 0; k < rc.K; ++k)
	{
		const u32 p = rc.p[k], q = rc.q[k], r2 = rc.r2[k];
		const u32 a0 = ref_red(d0, p);
		const u32 a1 = ref_mont(d1, r2, p, q);                       // d1 2^32
		const u32 a2 = ref_mont(ref_mont(d2, r2, p, q), r2, p, q);   // d2 2^64
		u32 r = ref_add(ref_add(a0, a1, p), a2, p);
		if (neg && r != 0) r = p - r;
		words[(size_t)k * n + i] = r;
	}
}

// Exact signed value from the K residues (mixed-radix Garner, leading digit
// balanced; kernel.cl:1231-1470), checked against the 96-bit normal form.
template <int K>
__global__ void k_import(const RefConst rc, const u32 * __restrict__ words, u32 * __restrict__ norm, u32 n, u32 * bad)
{
	const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	u32 u[K];
#pragma unroll
	for (int ii = K - 1; ii >= 0; --ii)
	{
		u32 v = words[(size_t)ii * n + i];
#pragma unroll
		for (int j = K - 1; j > ii; --j) v = ref_mont_c(ref_sub(v, u[j], rc.p[ii]), rc.gm[ii][j], rc.gmq[ii][j], rc.p[ii]);
		u[ii] = v;
	}
	const i32 i0 = (u[0] > (rc.p[0] >> 1)) ? (i32)(u[0] - rc.p[0]) : (i32)u[0];
	Big<K> V;
	{
		const i64 v01 = (i64)i0 * (i64)rc.p[1] + (i64)u[1];
		V.l[0] = (u32)v01; V.l[1] = (u32)((u64)v01 >> 32);
		const u32 sgn = (v01 < 0) ? 0xffffffffu : 0u;
#pragma unroll
		for (int l = 2; l < K; ++l) V.l[l] = sgn;
	}
#pragma unroll
	for (int l = 2; l < K; ++l) V = big_add_u32<K>(big_mul_u32<K>(V, rc.p[l]), u[l]);
	const u32 sgn = big_is_neg<K>(V) ? 0xffffffffu : 0u;
	u32 x[AB_NW];
#pragma unroll
	for (int l = 0; l < AB_NW; ++l) x[l] = (l < K) ? V.l[l] : sgn;
	bool fits = (K < AB_NW) || (((i32)x[2] < 0) == (sgn != 0));
#pragma unroll
	for (int l = AB_NW; l < K; ++l) fits = fits && (V.l[l] == sgn);
	if (!fits) atomicOr(bad, 1u);
#pragma unroll
	for (int l = 0; l < AB_NW; ++l) norm[(size_t)l * n + i] = x[l];
}

// ================================================================ mid pass
// The G levels between the column and the row levels (lengths above 2^20):
// with i = (h 2^G + m) R + c, global level LA + t works on bit G-1-t of m,
// block j = h 2^t + (m >> (G - t)).  One thread per (prime, h, c): 2^G words
// at stride R (consecutive threads, consecutive c).  Forward: [0, 4p) in and
// out; inverse: [0, 2p), twiddles -w^-1 (domain Q: the mirrored w).
template <int G, bool INV>
__global__ void __launch_bounds__(256) k_midpass(const RowJobs jobs, const TConst c)
{
	constexpr int M = 1 << G;
	const RowJob J = (blockIdx.y == 0) ? jobs.j[0] : jobs.j[1];
	const u32 cand = blockIdx.z;
	if (J.active != nullptr && J.active[cand] == 0u) return;
	const u32 R = c.R >> G;                      // row-pass row length
	const u32 per = c.H * R;
	const u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
	if (gid >= (u32)c.KP * per) return;
	const u32 k = gid / per, rem = gid - k * per, h = rem / R, col = rem - h * R;
	const u32 p = c.p[k], p2 = 2 * p;
	u32 * __restrict__ x = J.x + (size_t)cand * J.stride + (size_t)k * c.n + (size_t)h * M * R + col;
	const uint2 * __restrict__ w = J.w + (size_t)k * (c.n >> 1);
	const uint2 * __restrict__ wi = (J.wi != nullptr) ? J.wi + (size_t)k * (c.n >> 1) : nullptr;
	griddep_wait();
	griddep_launch();
	u32 v[M];
#pragma unroll
	for (int m = 0; m < M; ++m) v[m] = x[(size_t)m * R];
#pragma unroll
	for (int tt = 0; tt < G; ++tt)
	{
		const int t = INV ? G - 1 - tt : tt;
		const int half = M >> (t + 1);
		const u32 lvl = 1u << (c.LA + t);
#pragma unroll
		for (int blk = 0; blk < (1 << t); ++blk)
		{
			const u32 idx = lvl + (h << t) + (u32)blk;
			const uint2 wv = !INV ? __ldg(w + idx) : (wi != nullptr) ? __ldg(wi + idx) : __ldg(w + (3u * lvl - 1u - idx));
#pragma unroll
			for (int q = 0; q < half; ++q)
			{
				const int m0 = blk * 2 * half + q;
				if (INV) inv_bf(v[m0], v[m0 + half], wv.x, wv.y, p, p2);
				else fwd_bf(v[m0], v[m0 + half], wv.x, wv.y, p, p2);
			}
		}
	}
#pragma unroll
	for (int m = 0; m < M; ++m) x[(size_t)m * R] = v[m];
}

// ================================================================ host side
bool make_geometry(int ln, int lb_override, Geometry & g)
{
	if (ln < 6 || ln > 22) return false;
	const int L = ln - 1;
	// default split, measured on B200 for single transforms (us per squaring
	// over every split, ln 9..19): the row pass gets L - 2 levels up to 2^12
	// points, then 11 levels, and the column pass takes the rest (at most 6);
	// above 2^20 the row and column passes are full (13 and 6 levels) and the
	// mid pass takes the 1 or 2 levels left
	static const int DEFAULT_LB[23] = {0, 0, 0, 0, 0, 0, 4, 4, 5, 6, 7, 8, 9, 10, 10, 11, 11, 11, 11, 12, 13, 13, 13};
	int LB = (lb_override > 0) ? lb_override : DEFAULT_LB[ln];
	if (lb_override <= 0 && L - LB > 6 && ln <= 20) LB = L - 6;
	if (LB < 4 || LB > 13 || LB > L - 1) return false;
	const int LA = (L - LB < 6) ? L - LB : 6, G = L - LB - LA;
	if (G > 3) return false;
	g.ln = ln; g.LB = LB; g.LA = LA; g.G = G;
	g.H = 1u << LA; g.R = 1u << (LB + 1); g.HR = g.H << G; g.RC = g.R << G; g.C = CC;
	return true;
}

size_t colpass_smem(const Geometry & g, int KP)
{
	const size_t L = (size_t)KP - 1;
	return sizeof(u32) * ((size_t)KP * g.H * TW + (size_t)g.H * (TW / 4) * L) + sizeof(uint2) * 3 * (size_t)KP * g.H;
}

// The dynamic shared-memory limit of a kernel is a per-device setting: set it
// once for each device a process launches on (bit d of `done` = device d).
template <typename Kernel>
static cudaError_t allow_dynamic_smem(Kernel kernel, size_t smem, std::atomic<unsigned long long> & done)
{
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) return e;
	const unsigned long long bit = 1ull << (dev & 63);
	if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
	e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
	return e;
}

// Launch with programmatic stream serialization (see griddep_wait).
template <typename... P, typename... A>
static cudaError_t launch_pdl(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A &&... args)
{
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = smem;
	cfg.stream = s;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = AB_PDL;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

template <int LOG_R>
static cudaError_t rowpass_t(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s, int ncand)
{
	const size_t smem = RowCfg<LOG_R>::SMEM;
	static std::atomic<unsigned long long> attr_done{0};
	const cudaError_t e = allow_dynamic_smem(k_rowpass<LOG_R>, smem, attr_done);
	if (e != cudaSuccess) return e;
	if (ncand == 0) return cudaSuccess;      // set-up only (before a stream capture)
	const dim3 grid((unsigned)(c.KP * g.HR), (unsigned)njobs, (unsigned)ncand);
	return launch_pdl(k_rowpass<LOG_R>, grid, dim3(RowCfg<LOG_R>::NT), smem, s, jobs, c);
}

cudaError_t launch_rowpass(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s, int ncand)
{
	switch (g.LB + 1)
	{
	case 5: return rowpass_t<5>(g, c, jobs, njobs, s, ncand);
	case 6: return rowpass_t<6>(g, c, jobs, njobs, s, ncand);
	case 7: return rowpass_t<7>(g, c, jobs, njobs, s, ncand);
	case 8: return rowpass_t<8>(g, c, jobs, njobs, s, ncand);
	case 9: return rowpass_t<9>(g, c, jobs, njobs, s, ncand);
	case 10: return rowpass_t<10>(g, c, jobs, njobs, s, ncand);
	case 11: return rowpass_t<11>(g, c, jobs, njobs, s, ncand);
	case 12: return rowpass_t<12>(g, c, jobs, njobs, s, ncand);
	case 13: return rowpass_t<13>(g, c, jobs, njobs, s, ncand);
	case 14: return rowpass_t<14>(g, c, jobs, njobs, s, ncand);
	default: return cudaErrorInvalidValue;
	}
}

template <int G>
static cudaError_t midpass_t(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s, int ncand, bool inverse)
{
	const u32 threads = (u32)c.KP * g.H * g.R;
	const dim3 grid((threads + 255) / 256, (unsigned)njobs, (unsigned)ncand);
	if (inverse) return launch_pdl(k_midpass<G, true>, grid, dim3(256), 0, s, jobs, c);
	return launch_pdl(k_midpass<G, false>, grid, dim3(256), 0, s, jobs, c);
}

cudaError_t launch_midpass(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s, int ncand, bool inverse)
{
	if (ncand == 0) return cudaSuccess;
	switch (g.G)
	{
	case 1: return midpass_t<1>(g, c, jobs, njobs, s, ncand, inverse);
	case 2: return midpass_t<2>(g, c, jobs, njobs, s, ncand, inverse);
	case 3: return midpass_t<3>(g, c, jobs, njobs, s, ncand, inverse);
	default: return cudaErrorInvalidValue;
	}
}

template <int LOG_H, int K, int PCK>
static cudaError_t colpass_t(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s, int ncand)
{
	const size_t smem = colpass_smem(g, K + 1);
	static std::atomic<unsigned long long> attr_done{0};
	const cudaError_t e = allow_dynamic_smem(k_colpass<LOG_H, K, PCK>, smem, attr_done);
	if (e != cudaSuccess) return e;
	if (ncand == 0) return cudaSuccess;      // set-up only (before a stream capture)
	const dim3 grid(g.RC / CC, (unsigned)njobs, (unsigned)ncand);
	return launch_pdl(k_colpass<LOG_H, K, PCK>, grid, dim3(COL_THREADS), smem, s, jobs, c);
}

template <int K, int PCK>
static cudaError_t colpass_k(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s, int ncand)
{
	switch (g.LA)
	{
	case 1: return colpass_t<1, K, PCK>(g, c, jobs, njobs, s, ncand);
	case 2: return colpass_t<2, K, PCK>(g, c, jobs, njobs, s, ncand);
	case 3: return colpass_t<3, K, PCK>(g, c, jobs, njobs, s, ncand);
	case 4: return colpass_t<4, K, PCK>(g, c, jobs, njobs, s, ncand);
	case 5: return colpass_t<5, K, PCK>(g, c, jobs, njobs, s, ncand);
	case 6: return colpass_t<6, K, PCK>(g, c, jobs, njobs, s, ncand);
	default: return cudaErrorInvalidValue;
	}
}

cudaError_t launch_colpass(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s, int ncand)
{
	switch (c.K)
	{
	case 2: return colpass_k<2, 1>(g, c, jobs, njobs, s, ncand);
	case 3: return colpass_k<3, 2>(g, c, jobs, njobs, s, ncand);
	case 4: return colpass_k<4, 2>(g, c, jobs, njobs, s, ncand);
	case 5: return colpass_k<5, 4>(g, c, jobs, njobs, s, ncand);
	default: return cudaErrorInvalidValue;
	}
}

size_t fused_rowpass_smem(int log_r)
{
	return sizeof(u32) * (((size_t)1 << log_r) + ((size_t)1 << log_r) / 16);
}

cudaError_t launch_fused_rowpass(const FusedRowPass * d, const TConst * tcs, u32 ctas, size_t smem, cudaStream_t s)
{
	static std::atomic<unsigned long long> attr_done{0};
	static size_t set_smem = 0;
	if (smem > set_smem)
	{
		attr_done.store(0);
		set_smem = smem;
	}
	const cudaError_t e = allow_dynamic_smem(k_fused_rowpass, set_smem, attr_done);
	if (e != cudaSuccess || ctas == 0) return e;
	return launch_pdl(k_fused_rowpass, dim3(ctas), dim3(AB_FUSED_ROW_THREADS), smem, s, d, tcs);
}

cudaError_t launch_fused_colpass(const FusedColPass * d, const TConst * tcs, u32 ctas, size_t smem, cudaStream_t s)
{
	static std::atomic<unsigned long long> attr_done{0};
	static size_t set_smem = 0;
	if (smem > set_smem)
	{
		attr_done.store(0);
		set_smem = smem;
	}
	const cudaError_t e = allow_dynamic_smem(k_fused_colpass, set_smem, attr_done);
	if (e != cudaSuccess || ctas == 0) return e;
	return launch_pdl(k_fused_colpass, dim3(ctas), dim3(COL_THREADS), smem, s, d, tcs);
}

cudaError_t launch_export(const RefConst & rc, const u32 * norm, u32 * words, u32 n, cudaStream_t s)
{
	if (n == 0) return cudaSuccess;
	k_export<<<(n + 255) / 256, 256, 0, s>>>(rc, norm, words, n);
	return cudaGetLastError();
}

cudaError_t launch_import(const RefConst & rc, const u32 * words, u32 * norm, u32 n, u32 * bad, cudaStream_t s)
{
	if (n == 0) return cudaSuccess;
	const unsigned nb = (n + 255) / 256;
	switch (rc.K)
	{
	case 2: k_import<2><<<nb, 256, 0, s>>>(rc, words, norm, n, bad); break;
	case 3: k_import<3><<<nb, 256, 0, s>>>(rc, words, norm, n, bad); break;
	case 4: k_import<4><<<nb, 256, 0, s>>>(rc, words, norm, n, bad); break;
	case 5: k_import<5><<<nb, 256, 0, s>>>(rc, words, norm, n, bad); break;
	default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

} // namespace ab
