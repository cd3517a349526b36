// Device arithmetic for the multi-prime RNS transform (sm_100a).
//
// * Z/pZ for 32-bit primes p in (2^31, 2^32) with Montgomery multiplication,
//   R_M = 2^32, q = p^-1 mod 2^32 (same convention as src/transformGPU.h:21-59
//   and ocl/kernel.cl:122-149 of the reference: mont(a, b) = a*b*2^-32 mod p,
//   canonical result in [0, p)).
// * 32K-bit two's-complement integers (the reference's big_type,
//   ocl/kernel.cl:1212-1416: K=2 int64, 3 -> 96, 4 -> 128, 5 -> 160 bits),
//   held as K 32-bit limbs.
// * CRT (mixed-radix Garner) to the exact signed integer and the carry-digit
//   extraction rules (ocl/kernel.cl:1231-1559).
#pragma once
#include <cstdint>

typedef uint32_t u32;
typedef uint64_t u64;
typedef int32_t i32;
typedef int64_t i64;

#define AB_MAXK 5

// ---------------------------------------------------------------- Z/pZ
// a - b mod p: the borrow of the 32-bit subtraction becomes a mask m (0 or
// all ones) and the correction d - m p = d + p or d is one multiply-add, so
// the integer ALU pipe (the busiest unit of the NTT passes) does two
// operations and the multiply pipe one.
__device__ __forceinline__ u32 sub_mod(u32 a, u32 b, u32 p)
{
	const u64 d = (u64)a - b;
	const u32 m = (u32)(d >> 32);            // 0 or all ones (borrow)
	return (u32)d - m * p;
}

// a + b mod p = a - (p - b) mod p
__device__ __forceinline__ u32 add_mod(u32 a, u32 b, u32 p)
{
	return sub_mod(a, p - b, p);
}

// Final subtraction of the Montgomery products, in select form: measured
// faster here than the borrow-mask form (the product chain already loads the
// multiply pipe), and the form the products are validated with.
__device__ __forceinline__ u32 mont_sub(u32 h, u32 l, u32 p)
{
	const u32 d = h - l;
	return (h < l) ? d + p : d;
}

// a * b * 2^-32 mod p
__device__ __forceinline__ u32 mont_mul(u32 a, u32 b, u32 p, u32 q)
{
	const u64 t = (u64)a * b;
	const u32 m = (u32)t * q;
	return mont_sub((u32)(t >> 32), __umulhi(m, p), p);
}

// a * w * 2^-32 mod p with wq = w * q mod 2^32 precomputed (1 mul + 2 mulhi)
__device__ __forceinline__ u32 mont_mul_c(u32 a, u32 w, u32 wq, u32 p)
{
	return mont_sub(__umulhi(a, w), __umulhi(a * wq, p), p);
}

__device__ __forceinline__ u32 set_i32(i32 i, u32 p) { return (u32)i + ((i < 0) ? p : 0u); }

// Per-transform constants, passed by value to every kernel (lives in the
// kernel-parameter constant bank).
struct TConst
{
	u32 p[AB_MAXK], q[AB_MAXK], rsq[AB_MAXK];
	u32 norm[AB_MAXK];          // plain 2^-(ln-1) mod p
	u32 rbase[AB_MAXK];         // Montgomery form of 2^lbase: mont(v, rbase) = v * 2^lbase
	u32 rbase_pck[AB_MAXK];     // 2^(pck*lbase) mod p (plain)
	u32 gm[AB_MAXK][AB_MAXK];   // Montgomery form of P_j^-1 mod P_i (j > i)
	u32 gmq[AB_MAXK][AB_MAXK];  // gm * q_i mod 2^32
	u32 b2m[AB_MAXK], b2mq[AB_MAXK]; // Montgomery form of 2^(2*lbase) mod p (and *q)
	int K, pck, lbase, ln;
	u32 n;                      // 2^ln
	u32 R, H;                   // row length and row count of the 2-D NTT layout
	int LA, LB;                 // column levels, row levels
};

// Digit constants of one candidate (the digit size may differ between the
// candidates of a batch that share K and the NTT length).
struct CandConst
{
	int lbase;
	u32 rbase[AB_MAXK];         // Montgomery form of 2^lbase
	u32 rbase_pck[AB_MAXK];     // 2^(pck*lbase) mod p
};

// ---------------------------------------------------------------- big ints
template <int K>
struct Big
{
	u32 l[K];
};

template <int K>
__device__ __forceinline__ Big<K> big_zero()
{
	Big<K> r;
#pragma unroll
	for (int i = 0; i < K; ++i) r.l[i] = 0;
	return r;
}

template <int K>
__device__ __forceinline__ Big<K> big_from_i64(i64 v)
{
	Big<K> r;
	r.l[0] = (u32)v;
	r.l[1] = (u32)((u64)v >> 32);
	const u32 s = (v < 0) ? 0xffffffffu : 0u;
#pragma unroll
	for (int i = 2; i < K; ++i) r.l[i] = s;
	return r;
}

template <int K>
__device__ __forceinline__ Big<K> big_add(const Big<K> & a, const Big<K> & b)
{
	Big<K> r;
	u64 c = 0;
#pragma unroll
	for (int i = 0; i < K; ++i) { c += (u64)a.l[i] + b.l[i]; r.l[i] = (u32)c; c >>= 32; }
	return r;
}

template <int K>
__device__ __forceinline__ Big<K> big_sub(const Big<K> & a, const Big<K> & b)
{
	Big<K> r;
	u64 c = 1;
#pragma unroll
	for (int i = 0; i < K; ++i) { c += (u64)a.l[i] + (u64)(~b.l[i]); r.l[i] = (u32)c; c >>= 32; }
	return r;
}

template <int K>
__device__ __forceinline__ Big<K> big_neg(const Big<K> & a) { return big_sub<K>(big_zero<K>(), a); }

template <int K>
__device__ __forceinline__ Big<K> big_add_u32(const Big<K> & a, u32 v)
{
	Big<K> r;
	u64 c = v;
#pragma unroll
	for (int i = 0; i < K; ++i) { c += a.l[i]; r.l[i] = (u32)c; c >>= 32; }
	return r;
}

// a * y mod 2^(32K), y unsigned (sign-agnostic two's-complement product)
template <int K>
__device__ __forceinline__ Big<K> big_mul_u32(const Big<K> & a, u32 y)
{
	Big<K> r;
	u64 c = 0;
#pragma unroll
	for (int i = 0; i < K; ++i) { c += (u64)a.l[i] * y; r.l[i] = (u32)c; c >>= 32; }
	return r;
}

template <int K>
__device__ __forceinline__ bool big_is_neg(const Big<K> & a) { return (a.l[K - 1] >> 31) != 0; }

// arithmetic right shift by s, 0 < s < 32K.  s is the same in every thread
// (it derives from the digit size), so the limb move is a uniform branch and
// only the sub-limb part is a funnel shift.
template <int K>
__device__ __forceinline__ Big<K> big_sar(const Big<K> & a, int s)
{
	const u32 fill = big_is_neg<K>(a) ? 0xffffffffu : 0u;
	u32 t[K + 1];
#pragma unroll
	for (int i = 0; i < K; ++i) t[i] = a.l[i];
	t[K] = fill;
	int ws = s >> 5;
	while (ws > 0)
	{
#pragma unroll
		for (int i = 0; i < K; ++i) t[i] = t[i + 1];
		--ws;
	}
	const int bs = s & 31;
	Big<K> r;
	if (bs == 0)
	{
#pragma unroll
		for (int i = 0; i < K; ++i) r.l[i] = t[i];
	}
	else
	{
#pragma unroll
		for (int i = 0; i < K; ++i) r.l[i] = __funnelshift_r(t[i], t[i + 1], bs);
	}
	return r;
}

// v as K two's-complement limbs (v fits 32K bits)
template <int K>
__device__ __forceinline__ Big<K> big_from_i128(__int128 v)
{
	Big<K> r;
	const u32 s = (v < 0) ? 0xffffffffu : 0u;
#pragma unroll
	for (int i = 0; i < K; ++i) r.l[i] = (i < 4) ? (u32)((unsigned __int128)v >> (32 * i)) : s;
	return r;
}

template <int K>
__device__ __forceinline__ u64 big_low64(const Big<K> & a) { return (u64)a.l[0] | ((u64)a.l[1] << 32); }

// a >= 2^s (signed), s < 32K
template <int K>
__device__ __forceinline__ bool big_ge_pow2(const Big<K> & a, int s)
{
	if (big_is_neg<K>(a)) return false;
	const int w = s >> 5, b = s & 31;
	bool r = false;
#pragma unroll
	for (int i = 0; i < K; ++i)
	{
		if (i > w && a.l[i] != 0) r = true;
		if (i == w && (a.l[i] >> b) != 0) r = true;
	}
	return r;
}

// ---------------------------------------------------------------- CRT
// Exact signed integer V with V = r_k mod P_k (k < K): mixed-radix digits
// u_{K-1} .. u_0, the leading digit u_0 balanced into (-P0/2, P0/2].
template <int K>
__device__ __forceinline__ Big<K> garner(const TConst & c, const u32 (&r)[K])
{
	u32 u[K];
#pragma unroll
	for (int i = K - 1; i >= 0; --i)
	{
		u32 v = r[i];
#pragma unroll
		for (int j = K - 1; j > i; --j) v = mont_mul_c(sub_mod(v, u[j], c.p[i]), c.gm[i][j], c.gmq[i][j], c.p[i]);
		u[i] = v;
	}
	const i32 i0 = (u[0] > (c.p[0] >> 1)) ? (i32)(u[0] - c.p[0]) : (i32)u[0];
	if (K == 2)
	{
		const i64 v = (i64)i0 * (i64)c.p[1] + (i64)u[1];
		return big_from_i64<K>(v);
	}
	// i0 * P1 + u1 fits an int64; continue limb-wise for the remaining digits
	Big<K> V = big_from_i64<K>((i64)i0 * (i64)c.p[1] + (i64)u[1]);
#pragma unroll
	for (int i = 2; i < K; ++i) V = big_add_u32<K>(big_mul_u32<K>(V, c.p[i]), u[i]);
	return V;
}

// ---------------------------------------------------------------- digits
// Unsigned digits of the low pck*lbase bits of f, then f >>= pck*lbase
// (ocl/kernel.cl:1478-1537).
template <int K, int PCK>
__device__ __forceinline__ void extract_shift(Big<K> & f, int lb, u32 (&d)[PCK])
{
	const u32 bm = (1u << lb) - 1;
	const u64 low = big_low64<K>(f);
	if (PCK == 1)
	{
		d[0] = (u32)low & bm;
		f = big_sar<K>(f, lb);
	}
	else
	{
		const u64 r01 = low & (((u64)1 << (2 * lb)) - 1);
		d[0] = (u32)r01 & bm;
		d[1] = (u32)(r01 >> lb);
		f = big_sar<K>(f, 2 * lb);
		if (PCK == 4)
		{
			const u64 r23 = big_low64<K>(f) & (((u64)1 << (2 * lb)) - 1);
			d[2 % PCK] = (u32)r23 & bm;
			d[3 % PCK] = (u32)(r23 >> lb);
			f = big_sar<K>(f, 2 * lb);
		}
	}
}

// f + (d_0 + d_1 base + ... ) with unsigned digits
template <int K, int PCK>
__device__ __forceinline__ Big<K> add_digits(const Big<K> & f, int lb, const u32 (&d)[PCK])
{
	Big<K> t = big_zero<K>();
	if (PCK == 1) { t.l[0] = d[0]; }
	else
	{
		const u64 r01 = (u64)d[0] | ((u64)d[1] << lb);
		if (PCK == 2) { t.l[0] = (u32)r01; t.l[1] = (u32)(r01 >> 32); }
		else
		{
			const u64 r23 = (u64)d[2 % PCK] | ((u64)d[3 % PCK] << lb);
			// value = r01 + r23 * 2^(2 lb), 2 lb <= 62
			const int s = 2 * lb;
			const u64 lo = r01 | (r23 << s);
			const u64 hi = r23 >> (64 - s);
			t.l[0] = (u32)lo; t.l[1] = (u32)(lo >> 32);
			if (K > 2) t.l[2 % K] = (u32)hi;
			if (K > 3) t.l[3 % K] = (u32)(hi >> 32);
		}
	}
	return big_add<K>(f, t);
}

// Residues of D = sum_{l < PCK} d_l base^l (d_{PCK-1} signed, others in
// [0, base)) for each prime: Horner in the plain domain, top digit first
// (same value as encode() in ocl/kernel.cl:1474).
template <int K, int PCK>
__device__ __forceinline__ void encode_digits(const TConst & c, const u32 * rbase, i32 top, const u32 (&d)[PCK], u32 (&x)[K])
{
#pragma unroll
	for (int k = 0; k < K; ++k)
	{
		const u32 p = c.p[k];
		u32 v = set_i32(top, p);
		const u32 rb = rbase[k];
#pragma unroll
		for (int l = PCK - 2; l >= 0; --l)
		{
			// v = v * base + d_l  (base plain: mont(v, base*2^32) = v * base)
			v = mont_mul(v, rb, p, c.q[k]);
			v = add_mod(v, d[l], p);
		}
		x[k] = v;
	}
}
