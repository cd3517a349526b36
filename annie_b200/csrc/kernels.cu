// NTT passes of the modular-squaring engine, sm_100a.
//
// Mathematics (reference: ocl/kernel.cl and src/transformGPU.h of galloty/annie):
// a register holds, per prime p_k, n = 2^ln residues.  The forward transform
// is LN-1 radix-2 levels; the level with S polynomials maps each block of
// 2m = n/S coefficients mod (x^2m - c^2) to mod (x^m - c) and (x^m + c) with
// c = w[S + j] (j = block index, twiddle table in bit-reversed order,
// transformGPU.h:117-160).  The very first level takes plain residues and
// leaves Montgomery residues (lower half times rsq, upper half times
// w[0] = Montgomery(w[1]); kernel.cl:286-290).  The product of the resulting
// degree-1 polynomials is taken mod (x^2 -+ w[n/4 + q/2]) (kernel.cl:230-256),
// and the inverse levels undo the forward ones with the inverse twiddles
// (kernel.cl:218-228).  All values are canonical residues, so the results are
// bit-identical to the reference whatever the order of the butterflies.
//
// This file splits the n coefficients 2-D (row*R + col): the column pass owns
// the first LA levels (all H rows of 32 adjacent columns, all K primes, in
// shared memory) and the row pass owns the last LB levels (one row of one
// prime per CTA, 32 coefficients per thread in registers).
#include <atomic>

#include "kernels.h"

namespace ab
{

// ---------------------------------------------------------------- butterflies
__device__ __forceinline__ void fwd_bfly(u32 & x0, u32 & x1, u32 w, u32 wq, u32 p)
{
	const u32 t = mont_mul_c(x1, w, wq, p);
	x1 = sub_mod(x0, t, p);
	x0 = add_mod(x0, t, p);
}

__device__ __forceinline__ void inv_bfly(u32 & x0, u32 & x1, u32 wi, u32 wiq, u32 p)
{
	const u32 t = sub_mod(x0, x1, p);
	x0 = add_mod(x0, x1, p);
	x1 = mont_mul_c(t, wi, wiq, p);
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

// element of a stage with S group bits at bit b; the other bits come from
// o = tid + T*x (x selects one of the 16 / 2^S groups of the thread)
__device__ __forceinline__ u32 rp_elem(u32 tid, u32 T, int x, int S, int b, int g)
{
	const u32 o = tid + T * (u32)x;
	return (o & ((1u << b) - 1)) | ((u32)g << b) | ((o >> b) << (b + S));
}

// two pad words per 32: conflict-free for every stage layout, including the
// last one (lanes 2m, 2m+1 at elements 32m + {0,1} + 2g)
__device__ __forceinline__ u32 rp_pad(u32 e) { return e + ((e >> 5) << 1); }

template <int S, bool INV, bool SAVE>
__device__ __forceinline__ void rp_radix(u32 (&v)[RP_EPT], u32 tid, u32 T, int b, int LB, const u32 * __restrict__ w,
	u32 Hr, u32 p, u32 q, u32 (&w1)[8], u32 (&w1q)[8])
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
			const u32 * __restrict__ wl = w + ((Hr << t) + (ohi << (S - 1 - s)));
#pragma unroll
			for (int jh = 0; jh < (1 << (S - 1 - s)); ++jh)
			{
				const u32 wv = __ldg(wl + jh);
				const u32 wq = wv * q;
				if (SAVE && s == 0) { w1[jh] = wv; w1q[jh] = wq; }
#pragma unroll
				for (int gl = 0; gl < (1 << s); ++gl)
				{
					const int g = x * (1 << S) + (jh << (s + 1)) + gl;
					if (INV) inv_bfly(v[g], v[g + (1 << s)], wv, wq, p);
					else fwd_bfly(v[g], v[g + (1 << s)], wv, wq, p);
				}
			}
		}
	}
}

// Stage addressing: the 2^S words of a group are e0 + g 2^b.  In the padded
// shared layout they are pad(e0) + g D with D = 2^b + 2^(b-4) for b >= 5, and
// D = 2 for the last stage (b = 1, the group stays inside one 32-word block).
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
__device__ __forceinline__ void rp_pointwise(u32 (&v)[RP_EPT], const u32 * __restrict__ xp, bool is_mul, u32 tid, u32 NT,
	const u32 (&w1)[8], const u32 (&w1q)[8], u32 p, u32 q)
{
	// tid: virtual thread (its 16 words are the last-stage elements
	// 32*(tid>>1) + (tid&1) + 2g); NT: physical threads of the CTA (warp mask)
	const bool odd = (tid & 1) != 0;
	const unsigned mask = (NT >= 32) ? 0xffffffffu : ((1u << NT) - 1);
	u32 pv[RP_EPT];
	if (is_mul)
	{
#pragma unroll
		for (int i = 0; i < RP_EPT; ++i) pv[i] = __ldg(&xp[(tid & 1) + 2 * i + ((tid >> 1) << 5)]);
	}
#pragma unroll
	for (int i = 0; i < 8; ++i)
	{
		const u32 r = __shfl_xor_sync(mask, odd ? v[i] : v[8 + i], 1);
		const u32 x0 = odd ? r : v[i], x1 = odd ? v[8 + i] : r;
		const int slot = odd ? 8 + i : i;   // polynomial slot; parity = sign
		const u32 cw = odd ? w1[4 + (i >> 1)] : w1[i >> 1];
		const u32 cq = odd ? w1q[4 + (i >> 1)] : w1q[i >> 1];
		u32 t, y0, y1;
		if (is_mul)
		{
			const u32 rp2 = __shfl_xor_sync(mask, odd ? pv[i] : pv[8 + i], 1);
			const u32 p0 = odd ? rp2 : pv[i], p1 = odd ? pv[8 + i] : rp2;
			t = mont_mul_c(mont_mul(x1, p1, p, q), cw, cq, p);
			y1 = add_mod(mont_mul(x0, p1, p, q), mont_mul(p0, x1, p, q), p);
			y0 = mont_mul(x0, p0, p, q);
		}
		else
		{
			t = mont_mul_c(mont_mul(x1, x1, p, q), cw, cq, p);
			y1 = mont_mul(add_mod(x0, x0, p), x1, p, q);
			y0 = mont_mul(x0, x0, p, q);
		}
		y0 = ((slot & 1) == 0) ? add_mod(y0, t, p) : sub_mod(y0, t, p);
		const u32 r2 = __shfl_xor_sync(mask, odd ? y0 : y1, 1);
		if (odd) { v[8 + i] = y1; v[i] = r2; }
		else { v[i] = y0; v[8 + i] = r2; }
	}
}

// Physical threads of a row-pass CTA: 16 words per virtual thread, at most
// 256 threads, each running R / (16 * threads) rounds per stage.  The kernel
// is compiled for 4 CTAs per SM (at most 64 registers), so that the Q- and
// R-domain row passes, which run side by side on two streams, are resident
// together (measured: 4 % faster per squaring at 33.2 M bits than 3 per SM).
template <int LOG_R>
struct RowCfg
{
	static constexpr u32 T = (1u << LOG_R) / RP_EPT;             // virtual threads
	static constexpr u32 NT = (T < 256u) ? T : 256u;             // physical threads
	static constexpr u32 RND = T / NT;
};

template <int LOG_R>
__global__ void __launch_bounds__(RowCfg<LOG_R>::NT, 4) k_rowpass(const RowJobs jobs, const TConst c)
{
	constexpr int LB = LOG_R - 1;
	constexpr u32 T = RowCfg<LOG_R>::T, NT = RowCfg<LOG_R>::NT, RND = RowCfg<LOG_R>::RND;
	constexpr int NL = LB - 4;                                    // levels above the last stage
	constexpr int S0 = (NL % 4 == 0) ? 4 : NL % 4;                // first stage (when NL > 0)
	constexpr int NS = (NL == 0) ? 0 : 1 + (NL - S0) / 4;        // stages above the last
	constexpr int B0 = LB + 1 - S0;
	extern __shared__ __align__(16) u32 sm[];

	const RowJob J = (blockIdx.y == 0) ? jobs.j[0] : jobs.j[1];
	const u32 cand = blockIdx.z;
	if (J.active != nullptr && J.active[cand] == 0u) return;
	const size_t cofs = (size_t)cand * J.stride;
	const u32 k = blockIdx.x / c.H, r = blockIdx.x - k * c.H;
	const u32 p = c.p[k], q = c.q[k];
	u32 * __restrict__ x = J.x + cofs + (size_t)k * c.n + (size_t)r * (1u << LOG_R);
	const u32 * __restrict__ w = J.w + (size_t)k * c.n;
	const u32 * __restrict__ wi = w + (c.n >> 1);
	const u32 * __restrict__ xp = (J.mode == ROW_MUL) ? J.xp + cofs + (size_t)k * c.n + (size_t)r * (1u << LOG_R) : nullptr;
	const u32 Hr = c.H + r;
	const u32 tid = threadIdx.x;
	u32 v[RP_EPT];
	u32 w1[8], w1q[8];

	if constexpr (NS == 0)
	{
#pragma unroll 1
		for (u32 rr = 0; rr < RND; ++rr)
		{
			const u32 vt = tid + rr * NT;
			rp_load_global<4>(v, x, vt, T, 1);
			rp_radix<4, false, true>(v, vt, T, 1, LB, w, Hr, p, q, w1, w1q);
			if (J.mode != ROW_FWD_ONLY)
			{
				rp_pointwise(v, xp, J.mode == ROW_MUL, vt, NT, w1, w1q, p, q);
				rp_radix<4, true, false>(v, vt, T, 1, LB, wi, Hr, p, q, w1, w1q);
			}
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
			rp_load_global<S0>(v, x, vt, T, B0);
			rp_radix<S0, false, false>(v, vt, T, B0, LB, w, Hr, p, q, w1, w1q);
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
				rp_load_smem<4>(v, sm, vt, T, b);
				rp_radix<4, false, false>(v, vt, T, b, LB, w, Hr, p, q, w1, w1q);
				rp_store_smem<4>(v, sm, vt, T, b);
			}
		}
		__syncthreads();

		// ---- last stage (bits 4..1), pointwise, inverse last stage
#pragma unroll 1
		for (u32 rr = 0; rr < RND; ++rr)
		{
			const u32 vt = tid + rr * NT;
			rp_load_smem<4>(v, sm, vt, T, 1);
			rp_radix<4, false, true>(v, vt, T, 1, LB, w, Hr, p, q, w1, w1q);
			if (J.mode == ROW_FWD_ONLY)
			{
				rp_store_global<4>(v, x, vt, T, 1);
				continue;
			}
			rp_pointwise(v, xp, J.mode == ROW_MUL, vt, NT, w1, w1q, p, q);
			rp_radix<4, true, false>(v, vt, T, 1, LB, wi, Hr, p, q, w1, w1q);
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
				rp_load_smem<4>(v, sm, vt, T, b);
				rp_radix<4, true, false>(v, vt, T, b, LB, wi, Hr, p, q, w1, w1q);
				rp_store_smem<4>(v, sm, vt, T, b);
			}
		}
		__syncthreads();
#pragma unroll 1
		for (u32 rr = 0; rr < RND; ++rr)
		{
			const u32 vt = tid + rr * NT;
			rp_load_smem<S0>(v, sm, vt, T, B0);
			rp_radix<S0, true, false>(v, vt, T, B0, LB, wi, Hr, p, q, w1, w1q);
			rp_store_global<S0>(v, x, vt, T, B0);
		}
	}
}

// ================================================================ column pass
constexpr int CC = 32;  // own columns per CTA
constexpr int COL_THREADS = 384;
constexpr int TW = 40;  // tile row stride: own columns + up to 8 predecessor columns

// One radix-2^S step of the column transform (levels on row bits b..b+S-1)
// for one column of one prime: the 2^S rows that differ in those bits.
// Global level l (2^l polynomials) works on row bit LOG_H-1-l with twiddle
// w[2^l + j], j = row >> (LOG_H - l); level 0 of the forward direction takes
// plain residues (rsq / w[0] trick of kernel.cl:286-290).
template <int S, bool INV>
__device__ __forceinline__ void col_step(u32 * __restrict__ colp, int LOG_H, int b, u32 o, const u32 * __restrict__ tw,
	u32 p, u32 q, u32 rsq)
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
		const u32 * __restrict__ twl = tw + ((1u << lvl) + (ohi << (S - 1 - s)));
#pragma unroll
		for (int jh = 0; jh < (1 << (S - 1 - s)); ++jh)
		{
#pragma unroll
			for (int gl = 0; gl < (1 << s); ++gl)
			{
				const int g = (jh << (s + 1)) + gl;
				if (INV)
				{
					const u32 wv = twl[jh];
					inv_bfly(v[g], v[g + (1 << s)], wv, wv * q, p);
				}
				else if (lvl == 0)
				{
					const u32 w0 = tw[0];
					const u32 a0 = mont_mul_c(v[g], rsq, rsq * q, p), t = mont_mul_c(v[g + (1 << s)], w0, w0 * q, p);
					v[g] = add_mod(a0, t, p);
					v[g + (1 << s)] = sub_mod(a0, t, p);
				}
				else
				{
					const u32 wv = twl[jh];
					fwd_bfly(v[g], v[g + (1 << s)], wv, wv * q, p);
				}
			}
		}
	}
#pragma unroll
	for (int g = 0; g < (1 << S); ++g) base[g * D] = v[g];
}

// All LOG_H levels of the columns u in [u0, u0 + nu) of every prime, in place
// in the tile; stages of 3 levels (the remainder first in the forward order).
template <int LOG_H, int K, bool INV>
__device__ __forceinline__ void col_transform(u32 * tile, int u0, int nu, const u32 * twk, const TConst & c)
{
	constexpr int H = 1 << LOG_H;
	constexpr int SR = (LOG_H % 3 == 0) ? 3 : LOG_H % 3;       // top stage (row bits LOG_H-SR..LOG_H-1)
	constexpr int NST = 1 + (LOG_H - SR) / 3;
	const int tid = (int)threadIdx.x, NT = (int)blockDim.x;
#pragma unroll 1
	for (int st = 0; st < NST; ++st)
	{
		// forward: top stage first; inverse: bottom stage first
		const int idx = INV ? (NST - 1 - st) : st;
		const bool top = (idx == 0);
		const int b = top ? (LOG_H - SR) : (LOG_H - SR - 3 * idx);
		const int S = top ? SR : 3;
		const int ntask = K * nu * (H >> S);
		for (int task = tid; task < ntask; task += NT)
		{
			const int u = u0 + task % nu;
			const int rest = task / nu;
			const int o = rest % (H >> S), k = rest / (H >> S);
			u32 * colp = tile + (k * H) * TW + u;
			const u32 * tw = twk + k * H;
			if (S == 3) col_step<3, INV>(colp, LOG_H, b, (u32)o, tw, c.p[k], c.q[k], c.rsq[k]);
			else if (S == 2) col_step<2, INV>(colp, LOG_H, b, (u32)o, tw, c.p[k], c.q[k], c.rsq[k]);
			else col_step<1, INV>(colp, LOG_H, b, (u32)o, tw, c.p[k], c.q[k], c.rsq[k]);
		}
		__syncthreads();
	}
}

// Exact value of a balanced coefficient: unsigned digits e_0 .. e_{PCK-2} and
// the signed top digit, base 2^lb.
template <int K, int PCK>
__device__ __forceinline__ Big<K> digits_value(int lb, i32 top, const u32 (&e)[PCK])
{
	__int128 v = (__int128)top;
#pragma unroll
	for (int l = PCK - 2; l >= 0; --l) v = (v << lb) + (__int128)e[l];
	return big_from_i128<K>(v);
}

// Second carry phase for one group of 4 coefficients, in place in the tile:
// tp points at the group's first coefficient, plane l (digits) / k (residues)
// at tp + l * PS.  f = carry-in; each coefficient's digits are replaced by its
// balanced re-encoded residues (big: its exact value as K limbs); returns the
// top sub-digit of the last coefficient (kernel.cl:1582-1613).  The loop is
// rolled, so that the column pass body stays small enough for the
// instruction cache; a coefficient's digits are read before its residues
// overwrite them.
template <int K, int PCK>
__device__ __forceinline__ i32 carry_phase2(const TConst & c, int lb, const u32 * rbase, Big<K> f, u32 * tp, int PS, bool big, bool store)
{
	const i32 base = (i32)(1u << lb);
	auto put = [&](int j, i32 top, const u32 (&e)[PCK]) {
		u32 r[K];
		if (big)
		{
			const Big<K> v = digits_value<K, PCK>(lb, top, e);
#pragma unroll
			for (int k = 0; k < K; ++k) r[k] = v.l[k];
		}
		else encode_digits<K, PCK>(c, rbase, top, e, r);
		if (store)
		{
#pragma unroll
			for (int k = 0; k < K; ++k) tp[k * PS + j] = r[k];
		}
	};
#pragma unroll 1
	for (int j = 0; j < 3; ++j)
	{
		u32 d[PCK];
#pragma unroll
		for (int l = 0; l < PCK; ++l) d[l] = tp[l * PS + j];
		f = add_digits<K, PCK>(f, lb, d);
		u32 e[PCK];
		extract_shift<K, PCK>(f, lb, e);
		i32 top = (i32)e[PCK - 1];
		if (top >= base / 2) { top -= base; f = big_add_u32<K>(f, 1u); }
		put(j, top, e);
	}
	{
		u32 d[PCK];
#pragma unroll
		for (int l = 0; l < PCK; ++l) d[l] = tp[l * PS + 3];
		f = add_digits<K, PCK>(f, lb, d);
	}
	const u32 bm = (u32)base - 1;
	u32 e[PCK];
	i32 top;
	if (PCK == 1)
	{
		top = (i32)(i64)big_low64<K>(f);
	}
	else if (PCK == 2)
	{
		const i64 r01 = (i64)big_low64<K>(f);
		e[0] = (u32)r01 & bm;
		top = (i32)(r01 >> lb);
	}
	else
	{
		const u64 r01 = big_low64<K>(f) & (((u64)1 << (2 * lb)) - 1);
		e[0] = (u32)r01 & bm;
		e[1 % PCK] = (u32)(r01 >> lb);
		const Big<K> f23 = big_sar<K>(f, 2 * lb);
		const i64 r23 = (i64)big_low64<K>(f23);
		e[2 % PCK] = (u32)r23 & bm;
		top = (i32)(r23 >> lb);
	}
	put(3, top, e);
	return top;
}

// The same second phase unrolled over the 4 coefficients (faster for tall
// columns, LOG_H >= 5, where the body fits the instruction cache less badly
// than the lost parallelism costs): f = carry-in, d = the group's unsigned digits; writes the balanced re-encoded residues (BIG: the
// exact coefficient values as K limbs) and returns the top sub-digit of the
// last coefficient (kernel.cl:1582-1613).
template <int K, int PCK, bool BIG>
__device__ __forceinline__ i32 carry_phase2_unrolled(const TConst & c, int lb, const u32 * rbase, Big<K> f, const u32 (&d)[4][PCK], u32 (&res)[4][K])
{
	const i32 base = (i32)(1u << lb);
#pragma unroll
	for (int j = 0; j < 3; ++j)
	{
		f = add_digits<K, PCK>(f, lb, d[j]);
		u32 e[PCK];
		extract_shift<K, PCK>(f, lb, e);
		i32 top = (i32)e[PCK - 1];
		if (top >= base / 2) { top -= base; f = big_add_u32<K>(f, 1u); }
		if (BIG)
		{
			const Big<K> v = digits_value<K, PCK>(lb, top, e);
#pragma unroll
			for (int k = 0; k < K; ++k) res[j][k] = v.l[k];
		}
		else encode_digits<K, PCK>(c, rbase, top, e, res[j]);
	}
	f = add_digits<K, PCK>(f, lb, d[3]);
	const u32 bm = (u32)base - 1;
	u32 e[PCK];
	i32 top;
	if (PCK == 1)
	{
		top = (i32)(i64)big_low64<K>(f);
	}
	else if (PCK == 2)
	{
		const i64 r01 = (i64)big_low64<K>(f);
		e[0] = (u32)r01 & bm;
		top = (i32)(r01 >> lb);
	}
	else
	{
		const u64 r01 = big_low64<K>(f) & (((u64)1 << (2 * lb)) - 1);
		e[0] = (u32)r01 & bm;
		e[1 % PCK] = (u32)(r01 >> lb);
		const Big<K> f23 = big_sar<K>(f, 2 * lb);
		const i64 r23 = (i64)big_low64<K>(f23);
		e[2 % PCK] = (u32)r23 & bm;
		top = (i32)(r23 >> lb);
	}
	if (BIG)
	{
		const Big<K> v = digits_value<K, PCK>(lb, top, e);
#pragma unroll
		for (int k = 0; k < K; ++k) res[3][k] = v.l[k];
	}
	else encode_digits<K, PCK>(c, rbase, top, e, res[3]);
	return top;
}

template <int LOG_H, int K, int PCK>
__global__ void __launch_bounds__(COL_THREADS, 2) k_colpass(const ColJobs jobs, const TConst c)
{
	constexpr int H = 1 << LOG_H;
	// carry loops rolled over the 4 coefficients of a group for short columns,
	// unrolled for tall ones (measured: 12 % faster at LOG_H = 3 with K = 5,
	// equal at 4, 2 % slower at 5 and 6)
	constexpr bool ROLL = (LOG_H <= 4);
	extern __shared__ __align__(16) u32 sm[];
	u32 * const tile = sm;                       // [K][H][TW]
	u32 * const cw = tile + K * H * TW;          // [H][TW/4][K] carry-out words
	u32 * const twc = cw + H * (TW / 4) * K;     // [3][K][H] column twiddles
	__shared__ int decision;
	__shared__ CandConst cc;

	ColJob J = (blockIdx.y == 0) ? jobs.j[0] : jobs.j[1];
	const u32 cand = blockIdx.z;
	const u32 amul = (J.mult != nullptr) ? J.mult[cand] : J.a;
	if (amul == 0u) return;                       // inactive batch slot
	{
		const size_t cofs = (size_t)cand * J.stride;
		J.in += cofs;
		if (J.sub) J.sub += cofs;
		if (J.out_norm) J.out_norm += cofs;
		if (J.out_fwd[0]) J.out_fwd[0] += cofs;
		if (J.out_fwd[1]) J.out_fwd[1] += cofs;
		if (J.out_snap) J.out_snap = (J.snap_flag[cand] != 0u) ? J.out_snap + cofs : nullptr;
	}
	const u32 R = c.R, n = c.n;
	const int nb = (int)gridDim.x, b = (int)blockIdx.x;
	const u32 c0 = (u32)b * CC;
	const bool single = (nb == 1);
	// predecessor columns: the 4 left of the CTA (the last 4 of the previous row
	// for CTA 0); CTA 0 also takes the 4 before those when the mod R / mod Q
	// decision needs the final top coefficient
	const int E = (!J.transformed || single) ? 0 : ((b == 0 && J.lower != LOWER_NONE) ? 8 : 4);
	const int WU = CC + E, ng = WU / 4;
	const int tid = (int)threadIdx.x, NT = (int)blockDim.x;
	if (tid == 0)
	{
		if (J.cand != nullptr) cc = J.cand[cand];
		else
		{
			cc.lbase = c.lbase;
			for (int k = 0; k < AB_MAXK; ++k) { cc.rbase[k] = c.rbase[k]; cc.rbase_pck[k] = c.rbase_pck[k]; }
		}
	}

	auto gcol = [&](int u) -> u32 { return (u < E) ? ((b == 0) ? R - (u32)E + (u32)u : c0 - (u32)E + (u32)u) : c0 + (u32)(u - E); };

	// ---- load the tile and the column twiddles
	for (int idx = tid; idx < K * H * ng; idx += NT)
	{
		const int u4 = idx % ng, row = (idx / ng) % H, k = idx / (ng * H);
		const uint4 val = __ldg(reinterpret_cast<const uint4 *>(J.in + (size_t)k * n + (size_t)row * R + gcol(4 * u4)));
		*reinterpret_cast<uint4 *>(tile + (k * H + row) * TW + 4 * u4) = val;
	}
	for (int idx = tid; idx < K * H; idx += NT)
	{
		const int k = idx / H, i = idx % H;
		if (J.transformed) twc[idx] = J.w_in[(size_t)k * n + (n >> 1) + i];
		if (J.out_fwd[0] != nullptr) twc[K * H + idx] = J.w_out[0][(size_t)k * n + i];
		if (J.out_fwd[1] != nullptr) twc[2 * K * H + idx] = J.w_out[1][(size_t)k * n + i];
	}
	if (tid == 0) decision = 0;
	__syncthreads();
	const int lb = cc.lbase;

	if (J.transformed)
	{
		// ---- inverse column levels (all WU columns, K primes)
		col_transform<LOG_H, K, true>(tile, 0, WU, twc, c);

		// ---- carry phase 1: per group, unsigned digits + carry-out
		for (int idx = tid; idx < H * ng; idx += NT)
		{
			const int row = idx / ng, u4 = idx % ng;
			if (E == 8 && u4 == 0 && row != H - 1) continue;
			Big<K> f;
			if constexpr (ROLL)
			{
				// rolled over the 4 coefficients (code size); coefficient j's digits
				// overwrite its residues once they are read
				u32 * const tp = tile + row * TW + 4 * u4;
				const u32 * const sp = (J.sub != nullptr) ? J.sub + (size_t)row * R + gcol(4 * u4) : nullptr;
				f = big_zero<K>();
#pragma unroll 1
				for (int j = 0; j < 4; ++j)
				{
					u32 rr[K];
#pragma unroll
					for (int k = 0; k < K; ++k) rr[k] = mont_mul(tp[k * H * TW + j], c.norm[k], c.p[k], c.q[k]);
					const Big<K> V = garner<K>(c, rr);
					f = big_add<K>(f, (amul == 1u) ? V : big_mul_u32<K>(V, amul));
					if (sp != nullptr)
					{
#pragma unroll
						for (int k = 0; k < K; ++k) rr[k] = __ldg(sp + (size_t)k * n + j);
						Big<K> sv;
						if (J.sub_big)
						{
#pragma unroll
							for (int k = 0; k < K; ++k) sv.l[k] = rr[k];
						}
						else sv = garner<K>(c, rr);
						f = big_sub<K>(f, sv);
					}
					u32 dg[PCK];
					extract_shift<K, PCK>(f, lb, dg);
#pragma unroll
					for (int l = 0; l < PCK; ++l) tp[l * H * TW + j] = dg[l];
				}
			}
			else
			{
				u32 xv[K][4];
#pragma unroll
				for (int k = 0; k < K; ++k)
				{
					const uint4 t = *reinterpret_cast<const uint4 *>(tile + (k * H + row) * TW + 4 * u4);
					xv[k][0] = t.x; xv[k][1] = t.y; xv[k][2] = t.z; xv[k][3] = t.w;
				}
				u32 sv[K][4];
				if (J.sub != nullptr)
				{
#pragma unroll
					for (int k = 0; k < K; ++k)
					{
						const uint4 t = __ldg(reinterpret_cast<const uint4 *>(J.sub + (size_t)k * n + (size_t)row * R + gcol(4 * u4)));
						sv[k][0] = t.x; sv[k][1] = t.y; sv[k][2] = t.z; sv[k][3] = t.w;
					}
				}
				f = big_zero<K>();
				u32 dg[4][PCK];
#pragma unroll
				for (int j = 0; j < 4; ++j)
				{
					u32 rr[K];
#pragma unroll
					for (int k = 0; k < K; ++k) rr[k] = mont_mul(xv[k][j], c.norm[k], c.p[k], c.q[k]);
					const Big<K> V = garner<K>(c, rr);
					f = big_add<K>(f, (amul == 1u) ? V : big_mul_u32<K>(V, amul));
					if (J.sub != nullptr)
					{
						Big<K> s;
						if (J.sub_big)
						{
#pragma unroll
							for (int k = 0; k < K; ++k) s.l[k] = sv[k][j];
						}
						else
						{
#pragma unroll
							for (int k = 0; k < K; ++k) rr[k] = sv[k][j];
							s = garner<K>(c, rr);
						}
						f = big_sub<K>(f, s);
					}
					extract_shift<K, PCK>(f, lb, dg[j]);
				}
#pragma unroll
				for (int l = 0; l < PCK; ++l)
					*reinterpret_cast<uint4 *>(tile + (l * H + row) * TW + 4 * u4) = make_uint4(dg[0][l], dg[1][l], dg[2][l], dg[3][l]);
			}
#pragma unroll
			for (int k = 0; k < K; ++k) cw[(row * (TW / 4) + u4) * K + k] = f.l[k];
		}
		__syncthreads();

		// ---- carry phase 2: add the previous group's carry-out, balanced re-encode
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
			Big<K> f;
#pragma unroll
			for (int k = 0; k < K; ++k) f.l[k] = cw[(prow * (TW / 4) + pu4) * K + k];
			if (neg) f = big_neg<K>(f);
			i32 top;
			if constexpr (ROLL)
				top = carry_phase2<K, PCK>(c, lb, cc.rbase, f, tile + row * TW + 4 * u4, H * TW, J.out_big != 0, store);
			else
			{
				u32 dg[4][PCK];
#pragma unroll
				for (int l = 0; l < PCK; ++l)
				{
					const uint4 t = *reinterpret_cast<const uint4 *>(tile + (l * H + row) * TW + 4 * u4);
					dg[0][l] = t.x; dg[1][l] = t.y; dg[2][l] = t.z; dg[3][l] = t.w;
				}
				u32 res[4][K];
				top = J.out_big ? carry_phase2_unrolled<K, PCK, true>(c, lb, cc.rbase, f, dg, res)
				                : carry_phase2_unrolled<K, PCK, false>(c, lb, cc.rbase, f, dg, res);
				if (store)
				{
#pragma unroll
					for (int k = 0; k < K; ++k)
						*reinterpret_cast<uint4 *>(tile + (k * H + row) * TW + 4 * u4) = make_uint4(res[0][k], res[1][k], res[2][k], res[3][k]);
				}
			}
			const bool is_last = (row == H - 1) && (u4 == ng - 1) && (b == nb - 1);
			if ((is_last || !store) && top >= (i32)(1u << lb)) decision = 1;
		}
		__syncthreads();

		// ---- mod R (+2) / mod Q on the top and bottom coefficients (kernel.cl:1653-1683)
		if (J.lower != LOWER_NONE && tid < K)
		{
			const int k = tid;
			const u32 p = c.p[k];
			if (decision)
			{
				if (b == nb - 1)
				{
					u32 & t = tile[(k * H + H - 1) * TW + WU - 1];
					t = sub_mod(t, cc.rbase_pck[k], p);
				}
				if (b == 0)
				{
					u32 & t = tile[(k * H) * TW + E];
					t = sub_mod(t, set_i32((J.lower == LOWER_Q) ? 1 : -1, p), p);
				}
			}
			if (J.lower == LOWER_R_ADD2 && b == 0)
			{
				u32 & t = tile[(k * H) * TW + E];
				t = add_mod(t, 2u, p);
			}
		}
		__syncthreads();
	}

	// ---- outputs: normal form, then the first LA forward levels of the next
	// product, computed in place (the second domain reloads the normal form
	// from global memory)
	if (J.out_norm != nullptr || J.out_snap != nullptr)
	{
		for (int idx = tid; idx < K * H * (CC / 4); idx += NT)
		{
			const int u4 = idx % (CC / 4), row = (idx / (CC / 4)) % H, k = idx / ((CC / 4) * H);
			const uint4 val = *reinterpret_cast<const uint4 *>(tile + (k * H + row) * TW + E + 4 * u4);
			const size_t o = (size_t)k * n + (size_t)row * R + c0 + 4 * u4;
			if (J.out_norm) *reinterpret_cast<uint4 *>(J.out_norm + o) = val;
			if (J.out_snap) *reinterpret_cast<uint4 *>(J.out_snap + o) = val;
		}
		__syncthreads();
	}
	bool reload = false;
#pragma unroll 1
	for (int dom = 0; dom < 2; ++dom)
	{
		u32 * const out = (dom == 0) ? J.out_fwd[0] : J.out_fwd[1];
		if (out == nullptr) continue;
		if (reload)
		{
			__syncthreads();
			const u32 * src = J.transformed ? J.out_norm : J.in;
			for (int idx = tid; idx < K * H * (CC / 4); idx += NT)
			{
				const int u4 = idx % (CC / 4), row = (idx / (CC / 4)) % H, k = idx / ((CC / 4) * H);
				*reinterpret_cast<uint4 *>(tile + (k * H + row) * TW + E + 4 * u4) =
					*reinterpret_cast<const uint4 *>(src + (size_t)k * n + (size_t)row * R + c0 + 4 * u4);
			}
			__syncthreads();
		}
		col_transform<LOG_H, K, false>(tile, E, CC, twc + (1 + dom) * K * H, c);
		for (int idx = tid; idx < K * H * (CC / 4); idx += NT)
		{
			const int u4 = idx % (CC / 4), row = (idx / (CC / 4)) % H, k = idx / ((CC / 4) * H);
			*reinterpret_cast<uint4 *>(out + (size_t)k * n + (size_t)row * R + c0 + 4 * u4) =
				*reinterpret_cast<const uint4 *>(tile + (k * H + row) * TW + E + 4 * u4);
		}
		reload = true;
	}
}

// ================================================================ host side
bool make_geometry(int ln, int lb_override, Geometry & g)
{
	if (ln < 6 || ln > 20) return false;
	const int L = ln - 1;
	// default split, measured on B200 for single transforms (us per squaring
	// over every split, ln 9..19): the row pass gets L - 2 levels up to 2^12
	// points, then 11 levels, and the column pass takes the rest (at most 6)
	static const int DEFAULT_LB[21] = {0, 0, 0, 0, 0, 0, 4, 4, 5, 6, 7, 8, 9, 10, 10, 11, 11, 11, 11, 12, 13};
	int LB = (lb_override > 0) ? lb_override : DEFAULT_LB[ln];
	if (lb_override <= 0 && L - LB > 6) LB = L - 6;
	if (LB < 4 || LB > 13 || LB > L - 1 || L - LB > 6) return false;
	g.ln = ln; g.LB = LB; g.LA = L - LB;
	g.H = 1u << g.LA; g.R = 1u << (LB + 1); g.C = CC;
	return true;
}

size_t colpass_smem(const Geometry & g, int K)
{
	return sizeof(u32) * ((size_t)K * g.H * TW + (size_t)g.H * (TW / 4) * K + 3 * (size_t)K * g.H);
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

template <int LOG_R>
static cudaError_t rowpass_t(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s, int ncand)
{
	const u32 R = 1u << LOG_R;
	const size_t smem = sizeof(u32) * (R + R / 16);
	static std::atomic<unsigned long long> attr_done{0};
	const cudaError_t e = allow_dynamic_smem(k_rowpass<LOG_R>, smem, attr_done);
	if (e != cudaSuccess) return e;
	if (ncand == 0) return cudaSuccess;      // set-up only (before a stream capture)
	const dim3 grid((unsigned)(c.K * g.H), (unsigned)njobs, (unsigned)ncand);
	k_rowpass<LOG_R><<<grid, RowCfg<LOG_R>::NT, smem, s>>>(jobs, c);
	return cudaGetLastError();
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

template <int LOG_H, int K, int PCK>
static cudaError_t colpass_t(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s, int ncand)
{
	const size_t smem = colpass_smem(g, K);
	static std::atomic<unsigned long long> attr_done{0};
	const cudaError_t e = allow_dynamic_smem(k_colpass<LOG_H, K, PCK>, smem, attr_done);
	if (e != cudaSuccess) return e;
	if (ncand == 0) return cudaSuccess;      // set-up only (before a stream capture)
	const dim3 grid(g.R / CC, (unsigned)njobs, (unsigned)ncand);
	k_colpass<LOG_H, K, PCK><<<grid, COL_THREADS, smem, s>>>(jobs, c);
	return cudaGetLastError();
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

} // namespace ab
