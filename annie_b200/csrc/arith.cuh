// Device arithmetic of the modular-squaring engine (sm_100a).
//
// Two prime sets.
// * The transform primes (this engine's own choice): six primes p < 2^30 with
//   2^23 | p - 1.  A value mod p is kept lazily in [0, 2p) or [0, 4p) (4p <
//   2^32), so the NTT butterflies need no full reduction (Harvey's lazy
//   butterflies): a forward butterfly is a Shoup product (x w mod p with the
//   precomputed w' = floor(w 2^32 / p): 1 mulhi + 2 mul) and three adds.  A
//   class of the reference with K primes uses K + 1 of them: their product
//   exceeds the reference's prime product for every K, so every convolution
//   the reference computes exactly is exact here too.
// * The reference's primes (src/transformGPU.h:79-83, p in (2^31, 2^32)) are
//   only used to convert registers to and from the reference's register words
//   (its normal form is the residues, mod these primes, of each coefficient's
//   exact value; ocl/kernel.cl:1476-1559).
//
// A register's normal form is held as each coefficient's exact value: a
// 96-bit two's-complement integer in three 32-bit limbs.
#pragma once
#include <cstdint>

typedef uint32_t u32;
typedef uint64_t u64;
typedef int32_t i32;
typedef int64_t i64;

#define AB_MAXK 5          // primes of the reference's largest class
#define AB_MAXKP 6         // transform primes of that class
#define AB_NW 3            // words of a coefficient's exact value

// ---------------------------------------------------------------- transform primes
// x in [0, 4p) -> [0, 2p); p2 = 2p.  (x - 2p wraps above x when x < 2p.)
__device__ __forceinline__ u32 red2(u32 x, u32 p2) { return min(x, x - p2); }

// x w mod p in [0, 2p) for any x < 2^32 (Shoup: ws = floor(w 2^32 / p), w < p)
__device__ __forceinline__ u32 shoup(u32 x, u32 w, u32 ws, u32 p)
{
	const u32 q = __umulhi(x, ws);
	return x * w - q * p;
}

// a b 2^-32 mod p in (0, 2p) for a, b < 2p (Montgomery, pinv = p^-1 mod 2^32):
// a b - m p with m = (a b) pinv mod 2^32 is a multiple of 2^32, and
// a b / 2^32 < p, m p / 2^32 < p.
__device__ __forceinline__ u32 mont(u32 a, u32 b, u32 p, u32 pinv)
{
	const u32 lo = a * b, hi = __umulhi(a, b);
	return hi - __umulhi(lo * pinv, p) + p;
}

// Forward (decimation-in-time form) butterfly x0 +- w x1, inputs and outputs
// in [0, 4p).
__device__ __forceinline__ void fwd_bf(u32 & x0, u32 & x1, u32 w, u32 ws, u32 p, u32 p2)
{
	const u32 a = red2(x0, p2);
	const u32 t = shoup(x1, w, ws, p);
	x0 = a + t;
	x1 = a - t + p2;
}

// Inverse (Gentleman-Sande) butterfly with the stored twiddle v = -w^-1:
// x0 + x1 and (x1 - x0) v = (x0 - x1) w^-1; inputs and outputs in [0, 2p).
__device__ __forceinline__ void inv_bf(u32 & x0, u32 & x1, u32 v, u32 vs, u32 p, u32 p2)
{
	const u32 s = x0 + x1, d = x1 - x0 + p2;
	x0 = red2(s, p2);
	x1 = shoup(d, v, vs, p);
}

// ---------------------------------------------------------------- constants
// Per-transform constants, passed by value to every kernel (kernel-parameter
// constant bank).
struct TConst
{
	u32 p[AB_MAXKP], pinv[AB_MAXKP];
	u32 one_s[AB_MAXKP];                 // floor(2^32 / p): Shoup constant of 1
	u32 c32[AB_MAXKP], c32s[AB_MAXKP];   // 2^32 mod p and its Shoup constant
	u32 c64[AB_MAXKP], c64s[AB_MAXKP];   // 2^64 mod p
	u32 k95[AB_MAXKP];                   // -2^95 mod p (bias of the signed top limb)
	u32 crt[AB_MAXKP], crts[AB_MAXKP];   // (2/n) 2^32 (M/p)^-1 mod p: scale and CRT weight of the inverse output
	u32 fl[AB_MAXKP];                    // floor(2^60 / p): fixed-point 1/p of the CRT quotient estimate
	u32 mk[AB_MAXKP][AB_MAXK];           // (M/p) mod 2^(32 L), L = K limbs
	u32 negm[AB_MAXK];                   // -M mod 2^(32 L)
	int K, KP, pck, lbase, ln;           // reference primes K, transform primes KP = K + 1
	u32 n;                               // 2^ln
	u32 R, H;                            // column pass: row length and row count of the 2-D layout
	u32 HR;                              // row pass: rows (H 2^G) of 2^(LB+1) words
	int LA, LB, G;                       // column levels, row levels, mid levels (lengths above 2^20)
};

// Digit size of one candidate (candidates of a batch share K and the length).
struct CandConst
{
	int lbase;
};

// ---------------------------------------------------------------- big ints
template <int L>
struct Big
{
	u32 l[L];
};

template <int L>
__device__ __forceinline__ Big<L> big_zero()
{
	Big<L> r;
#pragma unroll
	for (int i = 0; i < L; ++i) r.l[i] = 0;
	return r;
}

template <int L>
__device__ __forceinline__ Big<L> big_add(const Big<L> & a, const Big<L> & b)
{
	Big<L> r;
	u64 c = 0;
#pragma unroll
	for (int i = 0; i < L; ++i) { c += (u64)a.l[i] + b.l[i]; r.l[i] = (u32)c; c >>= 32; }
	return r;
}

template <int L>
__device__ __forceinline__ Big<L> big_sub(const Big<L> & a, const Big<L> & b)
{
	Big<L> r;
	u64 c = 1;
#pragma unroll
	for (int i = 0; i < L; ++i) { c += (u64)a.l[i] + (u64)(~b.l[i]); r.l[i] = (u32)c; c >>= 32; }
	return r;
}

template <int L>
__device__ __forceinline__ Big<L> big_neg(const Big<L> & a) { return big_sub<L>(big_zero<L>(), a); }

template <int L>
__device__ __forceinline__ Big<L> big_add_u32(const Big<L> & a, u32 v)
{
	Big<L> r;
	u64 c = v;
#pragma unroll
	for (int i = 0; i < L; ++i) { c += a.l[i]; r.l[i] = (u32)c; c >>= 32; }
	return r;
}

// a * y mod 2^(32L), y unsigned (sign-agnostic two's-complement product)
template <int L>
__device__ __forceinline__ Big<L> big_mul_u32(const Big<L> & a, u32 y)
{
	Big<L> r;
	u64 c = 0;
#pragma unroll
	for (int i = 0; i < L; ++i) { c += (u64)a.l[i] * y; r.l[i] = (u32)c; c >>= 32; }
	return r;
}

template <int L>
__device__ __forceinline__ bool big_is_neg(const Big<L> & a) { return (a.l[L - 1] >> 31) != 0; }

// arithmetic right shift by s, 0 < s < 32L.  s is the same in every thread
// (it derives from the digit size), so the limb move is a uniform branch and
// only the sub-limb part is a funnel shift.
template <int L>
__device__ __forceinline__ Big<L> big_sar(const Big<L> & a, int s)
{
	const u32 fill = big_is_neg<L>(a) ? 0xffffffffu : 0u;
	u32 t[L + 1];
#pragma unroll
	for (int i = 0; i < L; ++i) t[i] = a.l[i];
	t[L] = fill;
	int ws = s >> 5;
	while (ws > 0)
	{
#pragma unroll
		for (int i = 0; i < L; ++i) t[i] = t[i + 1];
		--ws;
	}
	const int bs = s & 31;
	Big<L> r;
	if (bs == 0)
	{
#pragma unroll
		for (int i = 0; i < L; ++i) r.l[i] = t[i];
	}
	else
	{
#pragma unroll
		for (int i = 0; i < L; ++i) r.l[i] = __funnelshift_r(t[i], t[i + 1], bs);
	}
	return r;
}

// v as L two's-complement limbs (v fits 32L bits)
template <int L>
__device__ __forceinline__ Big<L> big_from_i128(__int128 v)
{
	Big<L> r;
	const u32 s = (v < 0) ? 0xffffffffu : 0u;
#pragma unroll
	for (int i = 0; i < L; ++i) r.l[i] = (i < 4) ? (u32)((unsigned __int128)v >> (32 * i)) : s;
	return r;
}

template <int L>
__device__ __forceinline__ u64 big_low64(const Big<L> & a) { return (u64)a.l[0] | ((u64)a.l[1] << 32); }

// a 96-bit exact value (three limbs) sign-extended or truncated to L limbs
template <int L>
__device__ __forceinline__ Big<L> big_from_exact(u32 d0, u32 d1, u32 d2)
{
	Big<L> r;
	const u32 s = ((i32)d2 < 0) ? 0xffffffffu : 0u;
#pragma unroll
	for (int i = 0; i < L; ++i) r.l[i] = (i == 0) ? d0 : (i == 1) ? d1 : (i == 2) ? d2 : s;
	return r;
}

// ---------------------------------------------------------------- CRT
// acc += y m (mod 2^(32L)): two carry chains, low halves then high halves.
template <int L>
__device__ __forceinline__ void big_mad_u32(u32 (&a)[L], u32 y, const u32 (&m)[AB_MAXK])
{
	if constexpr (L == 2)
	{
		asm("mad.lo.cc.u32 %0, %2, %3, %0;\n\t"
		    "madc.lo.u32 %1, %2, %4, %1;\n\t"
		    "mad.hi.u32 %1, %2, %3, %1;"
		    : "+r"(a[0]), "+r"(a[1]) : "r"(y), "r"(m[0]), "r"(m[1]));
	}
	else if constexpr (L == 3)
	{
		asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
		    "madc.lo.cc.u32 %1, %3, %5, %1;\n\t"
		    "madc.lo.u32 %2, %3, %6, %2;\n\t"
		    "mad.hi.cc.u32 %1, %3, %4, %1;\n\t"
		    "madc.hi.u32 %2, %3, %5, %2;"
		    : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]) : "r"(y), "r"(m[0]), "r"(m[1]), "r"(m[2]));
	}
	else if constexpr (L == 4)
	{
		asm("mad.lo.cc.u32 %0, %4, %5, %0;\n\t"
		    "madc.lo.cc.u32 %1, %4, %6, %1;\n\t"
		    "madc.lo.cc.u32 %2, %4, %7, %2;\n\t"
		    "madc.lo.u32 %3, %4, %8, %3;\n\t"
		    "mad.hi.cc.u32 %1, %4, %5, %1;\n\t"
		    "madc.hi.cc.u32 %2, %4, %6, %2;\n\t"
		    "madc.hi.u32 %3, %4, %7, %3;"
		    : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]) : "r"(y), "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]));
	}
	else
	{
		static_assert(L == 5, "2 to 5 limbs");
		asm("mad.lo.cc.u32 %0, %5, %6, %0;\n\t"
		    "madc.lo.cc.u32 %1, %5, %7, %1;\n\t"
		    "madc.lo.cc.u32 %2, %5, %8, %2;\n\t"
		    "madc.lo.cc.u32 %3, %5, %9, %3;\n\t"
		    "madc.lo.u32 %4, %5, %10, %4;\n\t"
		    "mad.hi.cc.u32 %1, %5, %6, %1;\n\t"
		    "madc.hi.cc.u32 %2, %5, %7, %2;\n\t"
		    "madc.hi.cc.u32 %3, %5, %8, %3;\n\t"
		    "madc.hi.u32 %4, %5, %9, %4;"
		    : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4])
		    : "r"(y), "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]));
	}
}

// Exact signed value V of a coefficient from its KP = L + 1 residues r_k in
// [0, 2p_k), which hold (n/2) 2^-32 V (the unnormalised inverse transform of a
// Montgomery pointwise product).  With y_k = r_k crt_k mod p_k in [0, p_k),
// V = sum y_k (M/p_k) - t M, t = round(sum y_k / p_k): the sum of fractions
// lies within |V|/M < 2^-18 of the integer t, so a 60-bit fixed-point estimate
// decides t exactly.  Computed mod 2^(32L), where V fits.
template <int L>
__device__ __forceinline__ Big<L> crt(const TConst & c, const u32 (&r)[L + 1])
{
	constexpr int KP = L + 1;
	u32 y[KP];
	u64 est = 0;
#pragma unroll
	for (int k = 0; k < KP; ++k)
	{
		const u32 p = c.p[k];
		const u32 v = shoup(r[k], c.crt[k], c.crts[k], p);
		y[k] = min(v, v - p);
		est += (u64)y[k] * c.fl[k];
	}
	const u32 t = (u32)((est + (1ull << 59)) >> 60);
	u32 a[L];
#pragma unroll
	for (int i = 0; i < L; ++i) a[i] = 0;
	big_mad_u32<L>(a, t, c.negm);
#pragma unroll
	for (int k = 0; k < KP; ++k) big_mad_u32<L>(a, y[k], c.mk[k]);
	Big<L> V;
#pragma unroll
	for (int i = 0; i < L; ++i) V.l[i] = a[i];
	return V;
}

// Residue in [0, 3p) of the exact value (d0, d1, d2) (two's complement): d0 +
// 2^32 d1 + 2^64 (d2 ^ 2^31) - 2^95.
__device__ __forceinline__ u32 encode_res(const TConst & c, int k, u32 d0, u32 d1, u32 d2u)
{
	const u32 p = c.p[k], p2 = 2 * p;
	const u32 a = d0 - __umulhi(d0, c.one_s[k]) * p;
	const u32 b = shoup(d1, c.c32[k], c.c32s[k], p);
	const u32 e = shoup(d2u, c.c64[k], c.c64s[k], p);
	u32 s = red2(a + b, p2);
	s = red2(s + e, p2);
	return s + c.k95[k];
}

// ---------------------------------------------------------------- digits
// Unsigned digits of the low pck*lbase bits of f, then f >>= pck*lbase
// (ocl/kernel.cl:1478-1537).
template <int L, int PCK>
__device__ __forceinline__ void extract_shift(Big<L> & f, int lb, u32 (&d)[PCK])
{
	const u32 bm = (1u << lb) - 1;
	const u64 low = big_low64<L>(f);
	if (PCK == 1)
	{
		d[0] = (u32)low & bm;
		f = big_sar<L>(f, lb);
	}
	else
	{
		const u64 r01 = low & (((u64)1 << (2 * lb)) - 1);
		d[0] = (u32)r01 & bm;
		d[1] = (u32)(r01 >> lb);
		f = big_sar<L>(f, 2 * lb);
		if (PCK == 4)
		{
			const u64 r23 = big_low64<L>(f) & (((u64)1 << (2 * lb)) - 1);
			d[2 % PCK] = (u32)r23 & bm;
			d[3 % PCK] = (u32)(r23 >> lb);
			f = big_sar<L>(f, 2 * lb);
		}
	}
}

// f + (d_0 + d_1 base + ... ) with unsigned digits
template <int L, int PCK>
__device__ __forceinline__ Big<L> add_digits(const Big<L> & f, int lb, const u32 (&d)[PCK])
{
	Big<L> t = big_zero<L>();
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
			if (L > 2) t.l[2 % L] = (u32)hi;
			if (L > 3) t.l[3 % L] = (u32)(hi >> 32);
		}
	}
	return big_add<L>(f, t);
}

// Exact value of a balanced coefficient (unsigned digits e_0 .. e_{PCK-2},
// signed top digit, base 2^lb) as three two's-complement limbs.
template <int PCK>
__device__ __forceinline__ void digits_exact(int lb, i32 top, const u32 (&e)[PCK], u32 & d0, u32 & d1, u32 & d2)
{
	__int128 v = (__int128)top;
#pragma unroll
	for (int l = PCK - 2; l >= 0; --l) v = (v << lb) + (__int128)e[l];
	const unsigned __int128 u = (unsigned __int128)v;
	d0 = (u32)u; d1 = (u32)(u >> 32); d2 = (u32)(u >> 64);
}

// ---------------------------------------------------------------- reference primes
// Montgomery arithmetic mod the reference's primes (p in (2^31, 2^32),
// canonical results; src/transformGPU.h:21-59), for the register-word
// conversions only.
struct RefConst
{
	u32 p[AB_MAXK], q[AB_MAXK];          // q = p^-1 mod 2^32
	u32 r2[AB_MAXK];                     // 2^64 mod p (Montgomery form of 2^32)
	u32 gm[AB_MAXK][AB_MAXK], gmq[AB_MAXK][AB_MAXK];   // Montgomery form of P_j^-1 mod P_i (j > i), and * q_i
	int K;
};

__device__ __forceinline__ u32 ref_sub(u32 a, u32 b, u32 p)
{
	const u32 d = a - b;
	return (a < b) ? d + p : d;
}

__device__ __forceinline__ u32 ref_mont_c(u32 a, u32 w, u32 wq, u32 p)
{
	return ref_sub(__umulhi(a, w), __umulhi(a * wq, p), p);
}

// x mod p, any u32 x (p > 2^31)
__device__ __forceinline__ u32 ref_red(u32 x, u32 p) { return (x >= p) ? x - p : x; }
