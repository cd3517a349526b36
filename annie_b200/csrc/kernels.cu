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

// shared-memory index with one pad word per 32: conflict-free for both the
// strided stage layouts and the 32-consecutive-per-thread layout
__device__ __forceinline__ u32 padx(u32 e) { return e + (e >> 5); }

// ================================================================ row pass
// Stage plan for a row of R = 2^(LB+1) words (levels t = 0..LB-1 touch bit
// LB-t of the in-row index): the last stage owns bits 4..1 plus the pair bit
// 0 (32 consecutive words per thread); the LB-4 levels above are split into
// stages of at most 5 levels.
template <int LB>
struct RowPlan
{
	static constexpr int NL = LB - 4;
	static constexpr int NS = (NL + 4) / 5;
	__host__ __device__ static constexpr int size(int i) { return (NS == 0) ? 0 : NL / NS + ((i < NL % NS) ? 1 : 0); }
	__host__ __device__ static constexpr int blo(int i)
	{
		int b = LB + 1;
		for (int k = 0; k <= i; ++k) b -= size(k);
		return b;
	}
};

// element of a non-last stage: group bits g (S of them) at bit BLO, the other
// bits from o = tid + T*x
template <int S, int BLO, u32 T>
__device__ __forceinline__ u32 stage_elem(u32 tid, int x, int g)
{
	const u32 o = tid + T * (u32)x;
	return (o & ((1u << BLO) - 1)) | ((u32)g << BLO) | ((o >> BLO) << (BLO + S));
}

template <int LB, int S, int BLO, bool INV>
__device__ __forceinline__ void row_stage(u32 (&v)[32], u32 tid, const u32 * __restrict__ w, u32 Hr, u32 p, u32 q)
{
	constexpr int G = 32 >> S;
	constexpr u32 T = (1u << (LB + 1)) / 32;
#pragma unroll
	for (int x = 0; x < G; ++x)
	{
		const u32 ohi = (tid + T * (u32)x) >> BLO;
#pragma unroll
		for (int ss = 0; ss < S; ++ss)
		{
			const int s = INV ? ss : (S - 1 - ss);
			const int t = LB - BLO - s;
#pragma unroll
			for (int jh = 0; jh < (1 << (S - 1 - s)); ++jh)
			{
				const u32 jj = (u32)jh + (ohi << (S - 1 - s));
				const u32 wv = __ldg(&w[(Hr << t) + jj]);
				const u32 wq = wv * q;
#pragma unroll
				for (int gl = 0; gl < (1 << s); ++gl)
				{
					const int g = (jh << (s + 1)) + gl;
					if (INV) inv_bfly(v[x * (1 << S) + g], v[x * (1 << S) + g + (1 << s)], wv, wq, p);
					else fwd_bfly(v[x * (1 << S) + g], v[x * (1 << S) + g + (1 << s)], wv, wq, p);
				}
			}
		}
	}
}

template <int S, int BLO, u32 T>
__device__ __forceinline__ void stage_load_smem(u32 (&v)[32], const u32 * sm, u32 tid)
{
#pragma unroll
	for (int x = 0; x < (32 >> S); ++x)
#pragma unroll
		for (int g = 0; g < (1 << S); ++g) v[x * (1 << S) + g] = sm[padx(stage_elem<S, BLO, T>(tid, x, g))];
}

template <int S, int BLO, u32 T>
__device__ __forceinline__ void stage_store_smem(const u32 (&v)[32], u32 * sm, u32 tid)
{
#pragma unroll
	for (int x = 0; x < (32 >> S); ++x)
#pragma unroll
		for (int g = 0; g < (1 << S); ++g) sm[padx(stage_elem<S, BLO, T>(tid, x, g))] = v[x * (1 << S) + g];
}

template <int S, int BLO, u32 T>
__device__ __forceinline__ void stage_load_global(u32 (&v)[32], const u32 * __restrict__ x, u32 tid)
{
#pragma unroll
	for (int xx = 0; xx < (32 >> S); ++xx)
#pragma unroll
		for (int g = 0; g < (1 << S); ++g) v[xx * (1 << S) + g] = x[stage_elem<S, BLO, T>(tid, xx, g)];
}

template <int S, int BLO, u32 T>
__device__ __forceinline__ void stage_store_global(const u32 (&v)[32], u32 * __restrict__ x, u32 tid)
{
#pragma unroll
	for (int xx = 0; xx < (32 >> S); ++xx)
#pragma unroll
		for (int g = 0; g < (1 << S); ++g) x[stage_elem<S, BLO, T>(tid, xx, g)] = v[xx * (1 << S) + g];
}

// last stage: v[i] = row element tid*32 + i; levels on bits 4..1
template <int LB, bool INV>
__device__ __forceinline__ void row_last(u32 (&v)[32], u32 tid, const u32 * __restrict__ w, u32 Hr, u32 p, u32 q,
	u32 (&w1)[8], u32 (&w1q)[8])
{
#pragma unroll
	for (int bb = 0; bb < 4; ++bb)
	{
		const int b = INV ? (1 + bb) : (4 - bb);
		const int t = LB - b;
#pragma unroll
		for (int jh = 0; jh < (16 >> b); ++jh)
		{
			const u32 jj = (tid << (4 - b)) + (u32)jh;
			const u32 wv = __ldg(&w[(Hr << t) + jj]);
			const u32 wq = wv * q;
			if (!INV && b == 1) { w1[jh] = wv; w1q[jh] = wq; }
#pragma unroll
			for (int gl = 0; gl < (1 << b); ++gl)
			{
				const int i = (jh << (b + 1)) + gl;
				if (INV) inv_bfly(v[i], v[i + (1 << b)], wv, wq, p);
				else fwd_bfly(v[i], v[i + (1 << b)], wv, wq, p);
			}
		}
	}
}

// pointwise product of the 16 degree-1 polynomials held by the thread
__device__ __forceinline__ void row_pointwise(u32 (&v)[32], const u32 * __restrict__ xp, bool is_mul,
	const u32 (&w1)[8], const u32 (&w1q)[8], u32 p, u32 q)
{
	u32 pv[32];
	if (is_mul)
	{
#pragma unroll
		for (int i = 0; i < 8; ++i)
		{
			const uint4 t = __ldg(reinterpret_cast<const uint4 *>(xp) + i);
			pv[4 * i] = t.x; pv[4 * i + 1] = t.y; pv[4 * i + 2] = t.z; pv[4 * i + 3] = t.w;
		}
	}
#pragma unroll
	for (int m = 0; m < 16; ++m)
	{
		const u32 x0 = v[2 * m], x1 = v[2 * m + 1];
		const u32 cw = w1[m >> 1], cq = w1q[m >> 1];
		u32 t, y0, y1;
		if (is_mul)
		{
			const u32 p0 = pv[2 * m], p1 = pv[2 * m + 1];
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
		v[2 * m] = ((m & 1) == 0) ? add_mod(y0, t, p) : sub_mod(y0, t, p);
		v[2 * m + 1] = y1;
	}
}

template <int LOG_R>
__global__ void __launch_bounds__((1 << LOG_R) / 32) k_rowpass(const RowJobs jobs, const TConst c)
{
	constexpr int LB = LOG_R - 1;
	constexpr u32 T = (1u << LOG_R) / 32;
	using P = RowPlan<LB>;
	extern __shared__ __align__(16) u32 sm[];

	const RowJob J = (blockIdx.y == 0) ? jobs.j[0] : jobs.j[1];
	const u32 k = blockIdx.x / c.H, r = blockIdx.x - k * c.H;
	const u32 p = c.p[k], q = c.q[k];
	u32 * __restrict__ x = J.x + (size_t)k * c.n + (size_t)r * (1u << LOG_R);
	const u32 * __restrict__ w = J.w + (size_t)k * c.n;
	const u32 * __restrict__ wi = w + (c.n >> 1);
	const u32 Hr = c.H + r;
	const u32 tid = threadIdx.x;
	u32 v[32];
	u32 w1[8], w1q[8];

	// ---- forward
	if constexpr (P::NS == 0)
	{
#pragma unroll
		for (int i = 0; i < 8; ++i)
		{
			const uint4 t = reinterpret_cast<const uint4 *>(x + tid * 32)[i];
			v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
		}
	}
	else
	{
		constexpr int S0 = P::size(0), B0 = P::blo(0);
		stage_load_global<S0, B0, T>(v, x, tid);
		row_stage<LB, S0, B0, false>(v, tid, w, Hr, p, q);
		stage_store_smem<S0, B0, T>(v, sm, tid);
		__syncthreads();
		if constexpr (P::NS >= 2)
		{
			constexpr int S1 = P::size(1), B1 = P::blo(1);
			stage_load_smem<S1, B1, T>(v, sm, tid);
			row_stage<LB, S1, B1, false>(v, tid, w, Hr, p, q);
			stage_store_smem<S1, B1, T>(v, sm, tid);
			__syncthreads();
		}
#pragma unroll
		for (int i = 0; i < 32; ++i) v[i] = sm[padx(tid * 32 + i)];
	}
	row_last<LB, false>(v, tid, w, Hr, p, q, w1, w1q);

	if (J.mode == ROW_FWD_ONLY)
	{
#pragma unroll
		for (int i = 0; i < 8; ++i)
			reinterpret_cast<uint4 *>(x + tid * 32)[i] = make_uint4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
		return;
	}

	// ---- pointwise
	row_pointwise(v, (J.mode == ROW_MUL) ? J.xp + (size_t)k * c.n + (size_t)r * (1u << LOG_R) + tid * 32 : nullptr,
		J.mode == ROW_MUL, w1, w1q, p, q);

	// ---- inverse
	row_last<LB, true>(v, tid, wi, Hr, p, q, w1, w1q);
	if constexpr (P::NS == 0)
	{
#pragma unroll
		for (int i = 0; i < 8; ++i)
			reinterpret_cast<uint4 *>(x + tid * 32)[i] = make_uint4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
	}
	else
	{
#pragma unroll
		for (int i = 0; i < 32; ++i) sm[padx(tid * 32 + i)] = v[i];
		__syncthreads();
		if constexpr (P::NS >= 2)
		{
			constexpr int S1 = P::size(1), B1 = P::blo(1);
			stage_load_smem<S1, B1, T>(v, sm, tid);
			row_stage<LB, S1, B1, true>(v, tid, wi, Hr, p, q);
			stage_store_smem<S1, B1, T>(v, sm, tid);
			__syncthreads();
		}
		constexpr int S0 = P::size(0), B0 = P::blo(0);
		stage_load_smem<S0, B0, T>(v, sm, tid);
		row_stage<LB, S0, B0, true>(v, tid, wi, Hr, p, q);
		stage_store_global<S0, B0, T>(v, x, tid);
	}
}

// ================================================================ column pass
constexpr int CC = 32;  // own columns per CTA
constexpr int TW = 40;  // tile row stride: own columns + up to 8 predecessor columns

template <int LOG_H>
__device__ __forceinline__ void col_inv(u32 (&v)[1 << LOG_H], const u32 * wi, u32 p, u32 q)
{
	constexpr int H = 1 << LOG_H;
#pragma unroll
	for (int S = H / 2; S >= 1; S /= 2)
	{
		const int m = H / (2 * S);
#pragma unroll
		for (int j = 0; j < S; ++j)
		{
			const u32 wv = wi[S + j], wq = wv * q;
#pragma unroll
			for (int i = 0; i < m; ++i) inv_bfly(v[2 * m * j + i], v[2 * m * j + i + m], wv, wq, p);
		}
	}
}

template <int LOG_H>
__device__ __forceinline__ void col_fwd(u32 (&v)[1 << LOG_H], const u32 * w, u32 p, u32 q, u32 rsq)
{
	constexpr int H = 1 << LOG_H;
	{
		const u32 w0 = w[0], w0q = w0 * q, rq = rsq * q;
#pragma unroll
		for (int i = 0; i < H / 2; ++i)
		{
			const u32 a = mont_mul_c(v[i], rsq, rq, p), t = mont_mul_c(v[i + H / 2], w0, w0q, p);
			v[i] = add_mod(a, t, p);
			v[i + H / 2] = sub_mod(a, t, p);
		}
	}
#pragma unroll
	for (int S = 2; S <= H / 2; S *= 2)
	{
		const int m = H / (2 * S);
#pragma unroll
		for (int j = 0; j < S; ++j)
		{
			const u32 wv = w[S + j], wq = wv * q;
#pragma unroll
			for (int i = 0; i < m; ++i) fwd_bfly(v[2 * m * j + i], v[2 * m * j + i + m], wv, wq, p);
		}
	}
}

// Second carry phase for one group of 4 coefficients: f = carry-in, d = the
// group's unsigned digits; writes the balanced re-encoded residues and returns
// the top sub-digit of the last coefficient (kernel.cl:1582-1613).
template <int K, int PCK>
__device__ __forceinline__ i32 carry_phase2(const TConst & c, Big<K> f, const u32 (&d)[4][PCK], u32 (&res)[4][K])
{
	const int lb = c.lbase;
	const i32 base = (i32)(1u << lb);
#pragma unroll
	for (int j = 0; j < 3; ++j)
	{
		f = add_digits<K, PCK>(f, lb, d[j]);
		u32 e[PCK];
		extract_shift<K, PCK>(f, lb, e);
		i32 top = (i32)e[PCK - 1];
		if (top >= base / 2) { top -= base; f = big_add_u32<K>(f, 1u); }
		encode_digits<K, PCK>(c, top, e, res[j]);
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
	encode_digits<K, PCK>(c, top, e, res[3]);
	return top;
}

template <int LOG_H, int K, int PCK>
__global__ void __launch_bounds__(256) k_colpass(const ColJobs jobs, const TConst c)
{
	constexpr int H = 1 << LOG_H;
	extern __shared__ __align__(16) u32 sm[];
	u32 * const tile = sm;                       // [K][H][TW]
	u32 * const cw = tile + K * H * TW;          // [H][TW/4][K] carry-out words
	u32 * const twc = cw + H * (TW / 4) * K;     // [3][K][H] column twiddles
	__shared__ int decision;

	const ColJob J = (blockIdx.y == 0) ? jobs.j[0] : jobs.j[1];
	const u32 R = c.R, n = c.n;
	const int nb = (int)gridDim.x, b = (int)blockIdx.x;
	const u32 c0 = (u32)b * CC;
	const bool single = (nb == 1);
	const int E = (!J.transformed || single) ? 0 : ((b == 0) ? 8 : 4);
	const int WU = CC + E, ng = WU / 4;
	const int tid = (int)threadIdx.x, NT = (int)blockDim.x;
	const int lb = c.lbase;

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

	if (J.transformed)
	{
		// ---- inverse column levels (all WU columns, K primes)
		for (int task = tid; task < K * WU; task += NT)
		{
			const int k = task / WU, u = task % WU;
			u32 v[H];
#pragma unroll
			for (int row = 0; row < H; ++row) v[row] = tile[(k * H + row) * TW + u];
			col_inv<LOG_H>(v, twc + k * H, c.p[k], c.q[k]);
#pragma unroll
			for (int row = 0; row < H; ++row) tile[(k * H + row) * TW + u] = v[row];
		}
		__syncthreads();

		// ---- carry phase 1: per group, unsigned digits + carry-out
		for (int idx = tid; idx < H * ng; idx += NT)
		{
			const int row = idx / ng, u4 = idx % ng;
			if (E == 8 && u4 == 0 && row != H - 1) continue;
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
			Big<K> f = big_zero<K>();
			u32 dg[4][PCK];
#pragma unroll
			for (int j = 0; j < 4; ++j)
			{
				u32 rr[K];
#pragma unroll
				for (int k = 0; k < K; ++k) rr[k] = mont_mul(xv[k][j], c.norm[k], c.p[k], c.q[k]);
				f = big_add<K>(f, big_mul_u32<K>(garner<K>(c, rr), J.a));
				if (J.sub != nullptr)
				{
#pragma unroll
					for (int k = 0; k < K; ++k) rr[k] = sv[k][j];
					f = big_sub<K>(f, garner<K>(c, rr));
				}
				extract_shift<K, PCK>(f, lb, dg[j]);
			}
#pragma unroll
			for (int l = 0; l < PCK; ++l)
				*reinterpret_cast<uint4 *>(tile + (l * H + row) * TW + 4 * u4) = make_uint4(dg[0][l], dg[1][l], dg[2][l], dg[3][l]);
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
				if (!(E == 8 && J.lower != LOWER_NONE)) continue;
				row = H - 1; u4 = 1; store = false;
			}
			else
			{
				row = idx / own_groups; u4 = E / 4 + idx % own_groups;
			}
			int prow = row, pu4 = u4 - 1;
			bool neg = false;
			if (store && u4 == E / 4 && E != 4)
			{
				pu4 = (E == 8) ? 1 : (ng - 1);
				if (row > 0) prow = row - 1;
				else { prow = H - 1; neg = (J.nega != 0); }
			}
			Big<K> f;
#pragma unroll
			for (int k = 0; k < K; ++k) f.l[k] = cw[(prow * (TW / 4) + pu4) * K + k];
			if (neg) f = big_neg<K>(f);
			u32 dg[4][PCK];
#pragma unroll
			for (int l = 0; l < PCK; ++l)
			{
				const uint4 t = *reinterpret_cast<const uint4 *>(tile + (l * H + row) * TW + 4 * u4);
				dg[0][l] = t.x; dg[1][l] = t.y; dg[2][l] = t.z; dg[3][l] = t.w;
			}
			u32 res[4][K];
			const i32 top = carry_phase2<K, PCK>(c, f, dg, res);
			const bool is_last = (row == H - 1) && (u4 == ng - 1) && (b == nb - 1);
			if ((is_last || !store) && top >= (i32)(1u << lb)) decision = 1;
			if (store)
			{
#pragma unroll
				for (int k = 0; k < K; ++k)
					*reinterpret_cast<uint4 *>(tile + (k * H + row) * TW + 4 * u4) = make_uint4(res[0][k], res[1][k], res[2][k], res[3][k]);
			}
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
					t = sub_mod(t, c.rbase_pck[k], p);
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

	// ---- outputs: normal form and the first LA forward levels of the next product
	if (J.out_norm != nullptr)
	{
		for (int idx = tid; idx < K * H * (CC / 4); idx += NT)
		{
			const int u4 = idx % (CC / 4), row = (idx / (CC / 4)) % H, k = idx / ((CC / 4) * H);
			const uint4 val = *reinterpret_cast<const uint4 *>(tile + (k * H + row) * TW + E + 4 * u4);
			*reinterpret_cast<uint4 *>(J.out_norm + (size_t)k * n + (size_t)row * R + c0 + 4 * u4) = val;
		}
	}
	const int nd = (J.out_fwd[0] != nullptr ? 1 : 0) + (J.out_fwd[1] != nullptr ? 1 : 0);
	for (int task = tid; task < nd * K * CC; task += NT)
	{
		int dom = task / (K * CC);
		if (J.out_fwd[0] == nullptr) dom = 1;
		const int k = (task / CC) % K, uc = task % CC;
		u32 v[H];
#pragma unroll
		for (int row = 0; row < H; ++row) v[row] = tile[(k * H + row) * TW + E + uc];
		col_fwd<LOG_H>(v, twc + (1 + dom) * K * H + k * H, c.p[k], c.q[k], c.rsq[k]);
		u32 * const out = J.out_fwd[dom] + (size_t)k * n + c0 + uc;
#pragma unroll
		for (int row = 0; row < H; ++row) out[(size_t)row * R] = v[row];
	}
}

// ================================================================ host side
bool make_geometry(int ln, int lb_override, Geometry & g)
{
	if (ln < 6 || ln > 20) return false;
	const int L = ln - 1;
	int LB = (lb_override > 0) ? lb_override : ((L - 1 < 12) ? L - 1 : 12);
	if (L - LB > 6) LB = L - 6;
	if (LB < 4 || LB > 13 || LB > L - 1) return false;
	g.ln = ln; g.LB = LB; g.LA = L - LB;
	g.H = 1u << g.LA; g.R = 1u << (LB + 1); g.C = CC;
	return true;
}

size_t colpass_smem(const Geometry & g, int K)
{
	return sizeof(u32) * ((size_t)K * g.H * TW + (size_t)g.H * (TW / 4) * K + 3 * (size_t)K * g.H);
}

template <int LOG_R>
static cudaError_t rowpass_t(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s)
{
	const u32 R = 1u << LOG_R;
	const size_t smem = sizeof(u32) * (R + R / 32);
	static bool attr = false;
	if (!attr)
	{
		cudaError_t e = cudaFuncSetAttribute(k_rowpass<LOG_R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		if (e != cudaSuccess) return e;
		attr = true;
	}
	const dim3 grid((unsigned)(c.K * g.H), (unsigned)njobs);
	k_rowpass<LOG_R><<<grid, R / 32, smem, s>>>(jobs, c);
	return cudaGetLastError();
}

cudaError_t launch_rowpass(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s)
{
	switch (g.LB + 1)
	{
	case 5: return rowpass_t<5>(g, c, jobs, njobs, s);
	case 6: return rowpass_t<6>(g, c, jobs, njobs, s);
	case 7: return rowpass_t<7>(g, c, jobs, njobs, s);
	case 8: return rowpass_t<8>(g, c, jobs, njobs, s);
	case 9: return rowpass_t<9>(g, c, jobs, njobs, s);
	case 10: return rowpass_t<10>(g, c, jobs, njobs, s);
	case 11: return rowpass_t<11>(g, c, jobs, njobs, s);
	case 12: return rowpass_t<12>(g, c, jobs, njobs, s);
	case 13: return rowpass_t<13>(g, c, jobs, njobs, s);
	case 14: return rowpass_t<14>(g, c, jobs, njobs, s);
	default: return cudaErrorInvalidValue;
	}
}

template <int LOG_H, int K, int PCK>
static cudaError_t colpass_t(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s)
{
	const size_t smem = colpass_smem(g, K);
	static bool attr = false;
	if (!attr)
	{
		cudaError_t e = cudaFuncSetAttribute(k_colpass<LOG_H, K, PCK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		if (e != cudaSuccess) return e;
		attr = true;
	}
	const dim3 grid(g.R / CC, (unsigned)njobs);
	k_colpass<LOG_H, K, PCK><<<grid, 256, smem, s>>>(jobs, c);
	return cudaGetLastError();
}

template <int K, int PCK>
static cudaError_t colpass_k(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s)
{
	switch (g.LA)
	{
	case 1: return colpass_t<1, K, PCK>(g, c, jobs, njobs, s);
	case 2: return colpass_t<2, K, PCK>(g, c, jobs, njobs, s);
	case 3: return colpass_t<3, K, PCK>(g, c, jobs, njobs, s);
	case 4: return colpass_t<4, K, PCK>(g, c, jobs, njobs, s);
	case 5: return colpass_t<5, K, PCK>(g, c, jobs, njobs, s);
	case 6: return colpass_t<6, K, PCK>(g, c, jobs, njobs, s);
	default: return cudaErrorInvalidValue;
	}
}

cudaError_t launch_colpass(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s)
{
	switch (c.K)
	{
	case 2: return colpass_k<2, 1>(g, c, jobs, njobs, s);
	case 3: return colpass_k<3, 2>(g, c, jobs, njobs, s);
	case 4: return colpass_k<4, 2>(g, c, jobs, njobs, s);
	case 5: return colpass_k<5, 4>(g, c, jobs, njobs, s);
	default: return cudaErrorInvalidValue;
	}
}

} // namespace ab
