/*
 * TEST INFRASTRUCTURE ONLY -- the oracle.  Never linked into the product.
 *
 * A plain-C restatement of the reference's modular-squaring engine
 * (galloty/annie: src/transformGPU.h + ocl/kernel.cl, with the CPU twin
 * src/transformCPU.h), written radix-2 and level by level so that it states
 * the mathematics rather than the reference's kernel schedule.  Every value it
 * produces is a canonical residue or an exact integer, so it is bit-comparable
 * with any correct implementation that uses the same parameters (K primes,
 * NTT length n = 2^ln, digit size lbase, packing pck).
 *
 * It is pinned against the reference's own transformCPU (compiled from the
 * reference sources into _ref/libannie_ref.so by the Makefile here): raw
 * register words after every square_mul must be equal for the K = 5, pck = 4
 * parameters transformCPU uses.  GMP (libgmp.so.10) provides the big-integer
 * set-up (N^-1 mod R, gcd) exactly as the reference uses it.
 *
 * Layout: a register is K planes of n uint32 residues, plane k at offset k*n.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "gmp.h"

typedef uint32_t u32;
typedef uint64_t u64;
typedef int32_t i32;
typedef int64_t i64;
typedef __int128 i128;
typedef unsigned __int128 u128;

/* The 14 primes P_k = c*2^e + 1 in (2^31, 2^32) and their primitive roots
   (src/transformGPU.h:79-89). */
#define PSIZE 14
static const u32 PRIME[PSIZE] = {
	(125u << 25) + 1, (243u << 24) + 1, (235u << 24) + 1, (29u << 27) + 1,
	(13u << 28) + 1, (193u << 24) + 1, (3u << 30) + 1, (43u << 26) + 1,
	(171u << 24) + 1, (81u << 25) + 1, (157u << 24) + 1, (151u << 24) + 1,
	(37u << 26) + 1, (17u << 27) + 1 };
static const u32 PROOT[PSIZE] = { 3, 7, 3, 3, 3, 3, 5, 3, 35, 5, 3, 3, 3, 3 };

/* ---- Z/pZ with Montgomery multiplication, R_M = 2^32 (transformGPU.h:21-114,
   kernel.cl:122-149).  q = p^-1 mod 2^32; mont(a, b) = a*b*2^-32 mod p. ---- */
typedef struct { u32 p, q, one, rsq; } zp;

static u32 inv_mod_2_32(u32 p) { u32 q = 1; for (int i = 0; i < 6; ++i) q *= 2 - p * q; return q; }
static u32 add_m(u32 a, u32 b, u32 p) { return a + b - ((a >= p - b) ? p : 0); }
static u32 sub_m(u32 a, u32 b, u32 p) { return a - b + ((a < b) ? p : 0); }
static u32 mont(u32 a, u32 b, const zp * z)
{
	const u64 t = (u64)a * b;
	const u32 m = (u32)t * z->q;
	const u32 mp = (u32)(((u64)m * z->p) >> 32);
	return sub_m((u32)(t >> 32), mp, z->p);
}
static zp zp_make(u32 p)
{
	zp z; z.p = p; z.q = inv_mod_2_32(p);
	z.one = (u32)(((u64)1 << 32) % p);
	z.rsq = (u32)(((u64)z.one * z.one) % p);
	return z;
}
static u32 to_mont(u32 a, const zp * z) { return mont(a, z->rsq, z); }
/* exponentiation in the Montgomery domain (transformGPU.h:61-73) */
static u32 pow_m(u32 x, u32 e, const zp * z)
{
	u32 r = z->one, y = x;
	while (e) { if (e & 1) r = mont(r, y, z); y = mont(y, y, z); e >>= 1; }
	return r;
}
static u32 inv_m(u32 x, const zp * z) { return pow_m(x, z->p - 2, z); }
static u32 primroot_n(int ln, int k, const zp * z) { return pow_m(to_mont(PROOT[k], z), (z->p - 1) >> ln, z); }
static u32 norm_m(int ln, const zp * z) { return z->p - ((z->p - 1) >> ln); }  /* plain 2^-ln */
static u32 set_i32(i32 i, u32 p) { return (u32)i + ((i < 0) ? p : 0); }

static size_t bitrev(size_t i, size_t n)
{
	size_t r = 0;
	for (size_t k = n, j = i; k > 1; k /= 2, j /= 2) r = (2 * r) | (j % 2);
	return r;
}

/* ---- twiddle tables (transformGPU.h:117-160): w[S + bitrev(j, S)] for the
   level with S polynomials, S = n/4 .. 1; w[0] = Montgomery form of w[1];
   inverse twiddles wi at offset n/2. ---- */
static void roots_R(u32 * w, int ln, int k, const zp * z)
{
	const size_t n = (size_t)1 << ln;
	u32 * wi = w + n / 2;
	u32 sr = primroot_n(ln - 1, k, z), sri = inv_m(sr, z);
	for (size_t s = n / 4; s >= 1; s /= 2)
	{
		u32 t = z->one, ti = z->one;
		for (size_t j = 0; j < s; ++j)
		{
			const size_t jr = bitrev(j, s);
			w[s + jr] = t; wi[s + jr] = ti;
			t = mont(t, sr, z); ti = mont(ti, sri, z);
		}
		sr = mont(sr, sr, z); sri = mont(sri, sri, z);
	}
	w[0] = to_mont(w[1], z);
	wi[0] = 0;
}

static void roots_Q(u32 * w, int ln, int k, const zp * z)
{
	const size_t n = (size_t)1 << ln;
	u32 * wi = w + n / 2;
	u32 sr2 = primroot_n(ln, k, z), sr2i = inv_m(sr2, z);
	for (size_t s = n / 4; s >= 1; s /= 2)
	{
		const u32 sr = mont(sr2, sr2, z), sri = mont(sr2i, sr2i, z);
		u32 t = sr2, ti = sr2i;
		for (size_t j = 0; j < s; ++j)
		{
			const size_t jr = bitrev(j, s);
			w[s + jr] = t; wi[s + jr] = ti;
			t = mont(t, sr, z); ti = mont(ti, sri, z);
		}
		sr2 = sr; sr2i = sri;
	}
	w[0] = to_mont(w[1], z);
	wi[0] = 0;
}

/* ---- 32K-bit two's-complement integers (the reference's big_type:
   kernel.cl:1212-1416; K=2: int64, 3: 96, 4: 128, 5: 160 bits). ---- */
typedef struct { u32 l[6]; } big;

static big big_norm(big a, int K) { for (int i = K; i < 6; ++i) a.l[i] = 0; return a; }
static big big_from_i128(i128 v, int K)
{
	big r; for (int i = 0; i < 6; ++i) { r.l[i] = (u32)v; v >>= 32; }
	return big_norm(r, K);
}
static big big_add(big a, big b, int K)
{
	big r; u64 c = 0;
	for (int i = 0; i < K; ++i) { c += (u64)a.l[i] + b.l[i]; r.l[i] = (u32)c; c >>= 32; }
	return big_norm(r, K);
}
static big big_neg(big a, int K)
{
	big r; u64 c = 1;
	for (int i = 0; i < K; ++i) { c += (u64)(~a.l[i]); r.l[i] = (u32)c; c >>= 32; }
	return big_norm(r, K);
}
static big big_sub(big a, big b, int K) { return big_add(a, big_neg(b, K), K); }
static big big_mul_u32(big a, u32 y, int K)
{
	big r; u64 c = 0;
	for (int i = 0; i < K; ++i) { c += (u64)a.l[i] * y; r.l[i] = (u32)c; c >>= 32; }
	return big_norm(r, K);
}
static int big_is_neg(big a, int K) { return (a.l[K - 1] >> 31) != 0; }
/* arithmetic shift right by s, 0 < s < 64 */
static big big_sar(big a, int s, int K)
{
	const u32 fill = big_is_neg(a, K) ? 0xffffffffu : 0u;
	u32 ext[8]; for (int i = 0; i < 8; ++i) ext[i] = (i < K) ? a.l[i] : fill;
	const int ws = s / 32, bs = s % 32;
	big r;
	for (int i = 0; i < K; ++i)
	{
		const u32 lo = ext[i + ws < 8 ? i + ws : 7], hi = ext[i + ws + 1 < 8 ? i + ws + 1 : 7];
		r.l[i] = (bs == 0) ? lo : (lo >> bs) | (hi << (32 - bs));
	}
	return big_norm(r, K);
}
static u64 big_low64(big a) { return (u64)a.l[0] | ((u64)a.l[1] << 32); }
/* x >= 2^s, s < 32K (kernel.cl:1225-1229, 1333-1371) */
static int big_ge_pow2(big a, int s, int K)
{
	if (big_is_neg(a, K)) return 0;
	for (int i = K * 32 - 1; i >= s; --i) if ((a.l[i / 32] >> (i % 32)) & 1) return 1;
	return 0;
}
/* for K = 2 the reference uses a plain int64 whose low word carries the
   low 32 bits: big_low64 covers both limbs. */

/* ---- the transform object ---- */
typedef struct
{
	int K, pck, ln, lbase;
	size_t n;
	int init_failed;
	zp z[PSIZE];
	u32 norm[PSIZE];
	u32 rbase_pck[PSIZE];       /* base^pck mod p (plain) */
	u32 inv_pj_pi[PSIZE][PSIZE];/* plain P_j^-1 mod P_i, j > i */
	u32 * wR; u32 * wQ;         /* per prime: n words (w || wi) */
	u32 * reg[8];               /* 0..2 public, 3 t_Q, 4 t, 5 one, 6 N_Q, 7 Ninv_R */
	mpz_t N, factor;
	big * cout;
	u32 * digits;               /* pck * n */
} oracle;

enum { R_TQ = 3, R_T = 4, R_ONE = 5, R_NQ = 6, R_NINVR = 7 };

static size_t get_s(size_t K) { int s = -1; for (size_t k = K - 1; k != 0; k /= 2) ++s; return (size_t)1 << s; }

/* ---- encode an integer into a register (transformGPU.h:323-360):
   coefficient i holds pck digits of lbase bits, residue = sum d_l base^l mod p. ---- */
static u32 read_bits(const u64 * x, size_t nl, size_t bit, int w)
{
	const size_t li = bit / 64; const int sh = (int)(bit % 64);
	const u64 lo = (li < nl) ? x[li] : 0, hi = (li + 1 < nl) ? x[li + 1] : 0;
	u64 r = lo >> sh; if (sh != 0) r |= hi << (64 - sh);
	return (u32)r & (u32)(((u64)1 << w) - 1);
}

static void set_mpz(oracle * o, u32 * reg, const mpz_t x)
{
	const size_t n = o->n, nl = mpz_size(x);
	const u64 * xl = (const u64 *)mpz_limbs_read(x);
	size_t bit = 0;
	for (size_t i = 0; i < n; ++i)
	{
		u128 d = 0;
		u32 dg[4];
		for (int l = 0; l < o->pck; ++l) { dg[l] = read_bits(xl, nl, bit, o->lbase); bit += (size_t)o->lbase; }
		for (int l = o->pck - 1; l >= 0; --l) d = (d << o->lbase) | dg[l];
		for (int k = 0; k < o->K; ++k) reg[(size_t)k * n + i] = (u32)(d % o->z[k].p);
	}
}

/* ---- NTT levels.  The level with S polynomials splits each block of
   2m = n/S coefficients mod (x^2m - c^2) into mod (x^m - c) and (x^m + c),
   c = w[S + j] (kernel.cl:206-228, 260-290). ---- */
static void fwd_level(u32 * x, const u32 * w, size_t n, size_t S, const zp * z)
{
	const size_t m = n / (2 * S);
	for (size_t j = 0; j < S; ++j)
	{
		u32 * b = x + 2 * m * j;
		if (S == 1)
		{
			/* input is plain: the upper half is multiplied by Montgomery(w[1]),
			   the lower half by rsq (kernel.cl:286-290, transformGPU.h:135) */
			for (size_t i = 0; i < m; ++i)
			{
				const u32 a = mont(b[i], z->rsq, z), t = mont(b[i + m], w[0], z);
				b[i] = add_m(a, t, z->p); b[i + m] = sub_m(a, t, z->p);
			}
		}
		else
		{
			const u32 c = w[S + j];
			for (size_t i = 0; i < m; ++i)
			{
				const u32 a = b[i], t = mont(b[i + m], c, z);
				b[i] = add_m(a, t, z->p); b[i + m] = sub_m(a, t, z->p);
			}
		}
	}
}

static void inv_level(u32 * x, const u32 * w, size_t n, size_t S, const zp * z)
{
	const size_t m = n / (2 * S);
	const u32 * wi = w + n / 2;
	for (size_t j = 0; j < S; ++j)
	{
		u32 * b = x + 2 * m * j;
		const u32 c = wi[S + j];
		for (size_t i = 0; i < m; ++i)
		{
			const u32 u = b[i], v = b[i + m];
			b[i] = add_m(u, v, z->p); b[i + m] = mont(sub_m(u, v, z->p), c, z);
		}
	}
}

static void fwd_full(oracle * o, u32 * x, const u32 * wtab)
{
	const size_t n = o->n;
	for (int k = 0; k < o->K; ++k)
		for (size_t S = 1; S <= n / 4; S *= 2) fwd_level(x + k * n, wtab + k * n, n, S, &o->z[k]);
}

static void inv_full(oracle * o, u32 * x, const u32 * wtab)
{
	const size_t n = o->n;
	for (int k = 0; k < o->K; ++k)
		for (size_t S = n / 4; S >= 1; S /= 2) inv_level(x + k * n, wtab + k * n, n, S, &o->z[k]);
}

/* pointwise product of degree-1 polynomials mod (x^2 - c), c = +-w[n/4 + q/2]
   (kernel.cl:230-256).  xp == NULL: square. */
static void pointwise(oracle * o, u32 * x, const u32 * xp, const u32 * wtab)
{
	const size_t n = o->n;
	for (int k = 0; k < o->K; ++k)
	{
		const zp * z = &o->z[k]; const u32 p = z->p;
		u32 * a = x + k * n; const u32 * b = xp ? xp + k * n : NULL;
		const u32 * w = wtab + k * n;
		for (size_t q = 0; q < n / 2; ++q)
		{
			const u32 c = w[n / 4 + q / 2];
			const u32 x0 = a[2 * q], x1 = a[2 * q + 1];
			u32 t, y0, y1;
			if (b == NULL)
			{
				t = mont(mont(x1, x1, z), c, z);
				y1 = mont(add_m(x0, x0, p), x1, z);
				y0 = mont(x0, x0, z);
			}
			else
			{
				const u32 p0 = b[2 * q], p1 = b[2 * q + 1];
				t = mont(mont(x1, p1, z), c, z);
				y1 = add_m(mont(x0, p1, z), mont(p0, x1, z), p);
				y0 = mont(x0, p0, z);
			}
			a[2 * q] = (q % 2 == 0) ? add_m(y0, t, p) : sub_m(y0, t, p);
			a[2 * q + 1] = y1;
		}
	}
}

/* ---- CRT: the exact signed integer V with V = r_k mod P_k, mixed-radix
   digits u_K-1 .. u_0 with the leading digit balanced (kernel.cl:1231-1470). ---- */
static big garner(oracle * o, const u32 * r)
{
	const int K = o->K;
	u32 u[PSIZE];
	for (int i = K - 1; i >= 0; --i)
	{
		const zp * z = &o->z[i];
		u32 v = r[i];
		for (int j = K - 1; j > i; --j) v = (u32)(((u64)sub_m(v, u[j] % z->p, z->p) * o->inv_pj_pi[i][j]) % z->p);
		u[i] = v;
	}
	const i32 i0 = (u[0] > o->z[0].p / 2) ? (i32)(u[0] - o->z[0].p) : (i32)u[0];
	big V = big_from_i128(i0, K);
	for (int i = 1; i < K; ++i) V = big_add(big_mul_u32(V, o->z[i].p, K), big_from_i128(u[i], K), K);
	return V;
}

/* digits of f: low pck*lbase bits, then f >>= pck*lbase (kernel.cl:1478-1537) */
static void extract_shift(oracle * o, big * f, u32 * d)
{
	const int K = o->K, lb = o->lbase;
	const u64 low = big_low64(*f);
	if (o->pck == 1) { d[0] = (u32)low & ((1u << lb) - 1); *f = big_sar(*f, lb, K); return; }
	const u64 r01 = low & (((u64)1 << (2 * lb)) - 1);
	d[0] = (u32)r01 & ((1u << lb) - 1); d[1] = (u32)(r01 >> lb);
	*f = big_sar(*f, 2 * lb, K);
	if (o->pck == 4)
	{
		const u64 r23 = big_low64(*f) & (((u64)1 << (2 * lb)) - 1);
		d[2] = (u32)r23 & ((1u << lb) - 1); d[3] = (u32)(r23 >> lb);
		*f = big_sar(*f, 2 * lb, K);
	}
}

static big pack_digits(oracle * o, const u32 * d)
{
	u128 v = 0;
	for (int l = o->pck - 1; l >= 0; --l) v = (v << o->lbase) | d[l];
	return big_from_i128((i128)v, o->K);
}

static void store_value(oracle * o, u32 * reg, size_t i, i128 D)
{
	for (int k = 0; k < o->K; ++k)
	{
		const u32 p = o->z[k].p;
		i128 m = D % (i128)p; if (m < 0) m += p;
		reg[(size_t)k * o->n + i] = (u32)m;
	}
}

/* balanced digits with carry into f (kernel.cl:1485-1546) */
static i128 extract_encode(oracle * o, big * f)
{
	u32 d[4]; extract_shift(o, f, d);
	const int pck = o->pck, lb = o->lbase;
	i32 top = (i32)d[pck - 1];
	if (top >= (i32)((1u << lb) / 2)) { top -= (i32)(1u << lb); *f = big_add(*f, big_from_i128(1, o->K), o->K); }
	i128 D = top;
	for (int l = pck - 2; l >= 0; --l) D = D * ((i128)1 << lb) + d[l];
	return D;
}

/* last coefficient of a group absorbs the rest unbalanced (kernel.cl:1493-1557) */
static i128 extract_encode_last(oracle * o, big f, i32 * top_out)
{
	const int lb = o->lbase; const u32 bm = (1u << lb) - 1;
	if (o->pck == 1) { const i32 r1 = (i32)(i64)big_low64(f); *top_out = r1; return r1; }
	if (o->pck == 2)
	{
		const i64 r01 = (i64)big_low64(f);
		const u32 r0 = (u32)r01 & bm; const i32 r1 = (i32)(r01 >> lb);
		*top_out = r1;
		return (i128)r1 * ((i128)1 << lb) + r0;
	}
	const u64 r01 = big_low64(f) & (((u64)1 << (2 * lb)) - 1);
	const u32 r0 = (u32)r01 & bm, r1 = (u32)(r01 >> lb);
	const big f23 = big_sar(f, 2 * lb, o->K);
	const i64 r23 = (i64)big_low64(f23);
	const u32 r2 = (u32)r23 & bm; const i32 r3 = (i32)(r23 >> lb);
	*top_out = r3;
	return (((i128)r3 * ((i128)1 << lb) + r2) * ((i128)1 << lb) + r1) * ((i128)1 << lb) + r0;
}

/* Carry propagation of one register after an inverse transform
   (kernel.cl:1561-1649 = transformCPU.h:1160-1211).  Groups of 4
   coefficients; phase 1 makes each group's unsigned digits and carry-out from
   its own values; phase 2 adds the previous group's carry-out (the last
   group's, negated for mod Q, for group 0) and re-encodes balanced digits.
   y != NULL subtracts y (normal-form register) before digit extraction. */
static void carry(oracle * o, u32 * x, u32 a, int nega, const u32 * y)
{
	const size_t n = o->n, G = n / 4; const int K = o->K, pck = o->pck;
	for (size_t g = 0; g < G; ++g)
	{
		big f = big_from_i128(0, K);
		for (size_t j = 0; j < 4; ++j)
		{
			const size_t c = 4 * g + j;
			u32 r[PSIZE];
			for (int k = 0; k < K; ++k) r[k] = mont(x[(size_t)k * n + c], o->norm[k], &o->z[k]);
			f = big_add(f, big_mul_u32(garner(o, r), a, K), K);
			if (y != NULL)
			{
				for (int k = 0; k < K; ++k) r[k] = y[(size_t)k * n + c];
				f = big_sub(f, garner(o, r), K);
			}
			extract_shift(o, &f, &o->digits[(size_t)pck * c]);
		}
		o->cout[g] = f;
	}
	for (size_t g = 0; g < G; ++g)
	{
		big f = (g > 0) ? o->cout[g - 1] : (nega ? big_neg(o->cout[G - 1], K) : o->cout[G - 1]);
		for (size_t j = 0; j < 3; ++j)
		{
			const size_t c = 4 * g + j;
			f = big_add(f, pack_digits(o, &o->digits[(size_t)pck * c]), K);
			store_value(o, x, c, extract_encode(o, &f));
		}
		const size_t c = 4 * g + 3;
		f = big_add(f, pack_digits(o, &o->digits[(size_t)pck * c]), K);
		i32 top; store_value(o, x, c, extract_encode_last(o, f, &top));
	}
}

/* If the top coefficient is >= base^pck subtract R (l0 = -1) or Q (l0 = 1)
   (kernel.cl:1653-1664). */
static void lower(oracle * o, u32 * x, i32 l0)
{
	const size_t n = o->n; const int K = o->K;
	u32 r[PSIZE]; for (int k = 0; k < K; ++k) r[k] = x[(size_t)k * n + n - 1];
	if (big_ge_pow2(garner(o, r), o->pck * o->lbase, K))
	{
		for (int k = 0; k < K; ++k)
		{
			const u32 p = o->z[k].p;
			x[(size_t)k * n + n - 1] = sub_m(x[(size_t)k * n + n - 1], o->rbase_pck[k], p);
			x[(size_t)k * n] = sub_m(x[(size_t)k * n], set_i32(l0, p), p);
		}
	}
}
static void mod_Q(oracle * o, u32 * x) { lower(o, x, 1); }
static void mod_R_add2(oracle * o, u32 * x)
{
	lower(o, x, -1);
	for (int k = 0; k < o->K; ++k) x[(size_t)k * o->n] = add_m(x[(size_t)k * o->n], 2, o->z[k].p);
}

static void copy_reg(oracle * o, u32 * d, const u32 * s) { if (d != s) memcpy(d, s, (size_t)o->K * o->n * 4); }

/* ---- MMGW sequences (transformGPU.h:523-568) ---- */
static void square_dom(oracle * o, u32 * x, const u32 * w) { fwd_full(o, x, w); pointwise(o, x, NULL, w); inv_full(o, x, w); }
static void mul_const(oracle * o, u32 * y, const u32 * xt, const u32 * w) { fwd_full(o, y, w); pointwise(o, y, xt, w); inv_full(o, y, w); }

static void reduce_mmgw(oracle * o, u32 * dst)
{
	mul_const(o, dst, o->reg[R_NINVR], o->wR);
	carry(o, dst, 1, 0, NULL);
	mod_R_add2(o, dst);
	mul_const(o, dst, o->reg[R_NQ], o->wQ);
	carry(o, dst, 1, 1, o->reg[R_TQ]);
	mod_Q(o, dst);
}

static void square_mmgw(oracle * o, u32 a)
{
	copy_reg(o, o->reg[R_TQ], o->reg[0]);
	square_dom(o, o->reg[R_TQ], o->wQ);
	carry(o, o->reg[R_TQ], a, 1, NULL);
	square_dom(o, o->reg[0], o->wR);
	carry(o, o->reg[0], a, 0, NULL);
	reduce_mmgw(o, o->reg[0]);
}

static void mul_mmgw(oracle * o, size_t dst, size_t src)
{
	u32 * t = o->reg[R_T];
	copy_reg(o, o->reg[R_TQ], o->reg[dst]);
	copy_reg(o, t, o->reg[src]);
	fwd_full(o, t, o->wQ);
	mul_const(o, o->reg[R_TQ], t, o->wQ);
	carry(o, o->reg[R_TQ], 1, 1, NULL);
	copy_reg(o, t, o->reg[src]);
	fwd_full(o, t, o->wR);
	mul_const(o, o->reg[dst], t, o->wR);
	carry(o, o->reg[dst], 1, 0, NULL);
	reduce_mmgw(o, o->reg[dst]);
}

/* ---- public C API (ctypes) ---- */

/* Parameter rule of the reference's GPU factory (transformGPU.h:798-857)
   when rule == 0, of transformCPU (transformCPU.h:1493-1533) when rule == 1. */
static void get_n_base(int * rln, int * rlbase, int pck, double log2_16aN, double log2_p_2a)
{
	for (int lbase = 31; lbase >= 2; --lbase)
	{
		int ln = 4; while ((double)(lbase * pck) * (1 << ln) < log2_16aN) ++ln;
		const int log2_base = lbase * pck;
		if (ln + 2 * log2_base < log2_p_2a) { *rln = ln; *rlbase = lbase; break; }
	}
}

int or_select_params(const uint64_t * nl, size_t ncount, int32_t a, int rule, int * K, int * pck, int * ln, int * lbase)
{
	mpz_t N; mpz_init(N); mpz_import(N, ncount, -1, 8, 0, 0, nl);
	long e_n; const double m_n = mpz_get_d_2exp(&e_n, N);
	mpz_clear(N);
	const double log2_16aN = log2(16.0 * a) + log2(m_n) + e_n;
	if (rule == 1)
	{
		double l = log2((double)PRIME[0]) + log2((double)PRIME[1]) + log2((double)PRIME[2]) + log2((double)PRIME[3]) - log2(2.0 * a);
		l += log2((double)PRIME[4]);
		*K = 5; *pck = 4; *ln = 0; *lbase = 0;
		get_n_base(ln, lbase, 4, log2_16aN, l);
		return 0;
	}
	double l = log2((double)PRIME[0]) - log2(2.0 * a);
	uint64_t c_min = (uint64_t)-1; size_t K_min = 0;
	for (size_t k = 2; k < 6; ++k)
	{
		l += log2((double)PRIME[k - 1]);
		const size_t s = get_s(k);
		int tln = 0, tlb = 0; get_n_base(&tln, &tlb, (int)s, log2_16aN, l);
		const uint64_t c = k * (uint64_t)(1u << tln) * (uint64_t)tln;
		if (c < c_min) { c_min = c; K_min = k; }
	}
	l = log2((double)PRIME[0]) - log2(2.0 * a);
	for (size_t k = 1; k < K_min; ++k) l += log2((double)PRIME[k]);
	*K = (int)K_min; *pck = (int)get_s(K_min); *ln = 0; *lbase = 0;
	get_n_base(ln, lbase, *pck, log2_16aN, l);
	return 0;
}

void * or_create(const uint64_t * nl, size_t ncount, int32_t a, int K, int ln, int lbase)
{
	(void)a;
	oracle * o = (oracle *)calloc(1, sizeof(oracle));
	o->K = K; o->pck = (int)get_s((size_t)K); o->ln = ln; o->lbase = lbase;
	const size_t n = (size_t)1 << ln; o->n = n;
	for (int k = 0; k < PSIZE; ++k) o->z[k] = zp_make(PRIME[k]);
	for (int k = 0; k < K; ++k)
	{
		const zp * z = &o->z[k];
		o->norm[k] = norm_m(ln - 1, z);
		u32 b = (u32)((1u << lbase) % z->p), bp = 1;
		for (int l = 0; l < o->pck; ++l) bp = (u32)(((u64)bp * b) % z->p);
		o->rbase_pck[k] = bp;
		for (int j = 0; j < K; ++j)
		{
			if (j <= k) continue;
			/* plain inverse of P_j mod P_k */
			u32 inv = inv_m(to_mont(PRIME[j] % z->p, z), z);
			o->inv_pj_pi[k][j] = mont(inv, 1, z);
		}
	}
	o->wR = (u32 *)malloc((size_t)K * n * 4); o->wQ = (u32 *)malloc((size_t)K * n * 4);
	for (int k = 0; k < K; ++k) { roots_R(o->wR + k * n, ln, k, &o->z[k]); roots_Q(o->wQ + k * n, ln, k, &o->z[k]); }
	for (int r = 0; r < 8; ++r) o->reg[r] = (u32 *)calloc((size_t)K * n, 4);
	o->cout = (big *)malloc((n / 4) * sizeof(big));
	o->digits = (u32 *)malloc((size_t)o->pck * n * 4);

	mpz_inits(o->N, o->factor, NULL);
	mpz_import(o->N, ncount, -1, 8, 0, 0, nl);
	mpz_t R, t; mpz_inits(R, t, NULL);
	mpz_set_ui(R, 1); mpz_mul_2exp(R, R, (mp_bitcnt_t)o->pck * lbase << ln); mpz_sub_ui(R, R, 1);
	if (mpz_invert(t, o->N, R) == 0)
	{
		mpz_gcd(o->factor, o->N, R);
		o->init_failed = 1;
		mpz_clears(R, t, NULL);
		return o;
	}
	set_mpz(o, o->reg[R_NQ], o->N); fwd_full(o, o->reg[R_NQ], o->wQ);
	set_mpz(o, o->reg[R_NINVR], t); fwd_full(o, o->reg[R_NINVR], o->wR);
	mpz_mod(t, R, o->N);
	if (mpz_odd_p(t)) mpz_add(t, t, o->N);
	mpz_fdiv_q_2exp(t, t, 1);
	set_mpz(o, o->reg[R_ONE], t);
	mpz_clears(R, t, NULL);
	return o;
}

void or_destroy(void * h)
{
	oracle * o = (oracle *)h;
	for (int r = 0; r < 8; ++r) free(o->reg[r]);
	free(o->wR); free(o->wQ); free(o->cout); free(o->digits);
	mpz_clears(o->N, o->factor, NULL);
	free(o);
}

int or_init_failed(void * h) { return ((oracle *)h)->init_failed; }
void or_set1(void * h) { oracle * o = (oracle *)h; copy_reg(o, o->reg[0], o->reg[R_ONE]); }
void or_copy(void * h, size_t dst, size_t src) { oracle * o = (oracle *)h; copy_reg(o, o->reg[dst], o->reg[src]); }
void or_square_mul(void * h, int32_t a) { square_mmgw((oracle *)h, (u32)a); }
void or_mul(void * h, size_t dst, size_t src) { mul_mmgw((oracle *)h, dst, src); }

/* register words, prime-major (reg 0..7) */
void or_read_reg(void * h, size_t r, uint32_t * out) { oracle * o = (oracle *)h; memcpy(out, o->reg[r], (size_t)o->K * o->n * 4); }
void or_write_reg(void * h, size_t r, const uint32_t * in) { oracle * o = (oracle *)h; memcpy(o->reg[r], in, (size_t)o->K * o->n * 4); }
void or_read_roots(void * h, int domain_q, uint32_t * out) { oracle * o = (oracle *)h; memcpy(out, domain_q ? o->wQ : o->wR, (size_t)o->K * o->n * 4); }

/* kernel-level pieces on a caller array of K*n words */
void or_fwd_full(void * h, int domain_q, uint32_t * x) { oracle * o = (oracle *)h; fwd_full(o, x, domain_q ? o->wQ : o->wR); }
void or_fwd_levels(void * h, int domain_q, uint32_t * x, int lv_from, int lv_to)
{
	oracle * o = (oracle *)h; const u32 * w = domain_q ? o->wQ : o->wR;
	for (int k = 0; k < o->K; ++k)
		for (int lv = lv_from; lv < lv_to; ++lv) fwd_level(x + k * o->n, w + k * o->n, o->n, (size_t)1 << lv, &o->z[k]);
}
void or_inv_levels(void * h, int domain_q, uint32_t * x, int lv_from, int lv_to)
{
	oracle * o = (oracle *)h; const u32 * w = domain_q ? o->wQ : o->wR;
	for (int k = 0; k < o->K; ++k)
		for (int lv = lv_to - 1; lv >= lv_from; --lv) inv_level(x + k * o->n, w + k * o->n, o->n, (size_t)1 << lv, &o->z[k]);
}
void or_pointwise(void * h, int domain_q, uint32_t * x, const uint32_t * xp) { oracle * o = (oracle *)h; pointwise(o, x, xp, domain_q ? o->wQ : o->wR); }
void or_inv_full(void * h, int domain_q, uint32_t * x) { oracle * o = (oracle *)h; inv_full(o, x, domain_q ? o->wQ : o->wR); }
/* lower_mode: 0 none, 1 mod_R_add2, 2 mod_Q */
void or_carry(void * h, uint32_t * x, uint32_t a, int nega, const uint32_t * y, int lower_mode)
{
	oracle * o = (oracle *)h;
	carry(o, x, a, nega, y);
	if (lower_mode == 1) mod_R_add2(o, x);
	else if (lower_mode == 2) mod_Q(o, x);
}

/* z = r_src mod N (transformGPU.h:576-586, 362-445); returns limb count. */
long or_get(void * h, size_t src, uint64_t * out, size_t cap)
{
	oracle * o = (oracle *)h;
	const size_t n = o->n; const int pck = o->pck, lb = o->lbase;
	u32 * t = o->reg[R_T];
	copy_reg(o, o->reg[R_TQ], o->reg[src]);
	copy_reg(o, t, o->reg[src]);
	reduce_mmgw(o, t);
	const size_t nbits = (size_t)pck * lb * n, nlimbs = nbits / 64 + 2;
	u64 * y = (u64 *)calloc(nlimbs, 8);
	i128 f = 0; size_t bit = 0;
	for (size_t i = 0; i < n; ++i)
	{
		/* Garner over the first pck primes only (transformGPU.h:182-260) */
		u32 u[4];
		for (int ii = pck - 1; ii >= 0; --ii)
		{
			const zp * z = &o->z[ii];
			u32 v = t[(size_t)ii * n + i];
			for (int j = pck - 1; j > ii; --j) v = (u32)(((u64)sub_m(v, u[j] % z->p, z->p) * o->inv_pj_pi[ii][j]) % z->p);
			u[ii] = v;
		}
		const i32 i0 = (u[0] > o->z[0].p / 2) ? (i32)(u[0] - o->z[0].p) : (i32)u[0];
		i128 D = i0;
		for (int ii = 1; ii < pck; ++ii) D = D * o->z[ii].p + u[ii];
		f += D;
		for (int l = 0; l < pck; ++l)
		{
			const u64 r = (u64)(f & (((i128)1 << lb) - 1));
			const size_t li = bit / 64; const int sh = (int)(bit % 64);
			y[li] |= r << sh; if (sh != 0 && sh + lb > 64) y[li + 1] |= r >> (64 - sh);
			f >>= lb; bit += (size_t)lb;
		}
	}
	mpz_t Y, F; mpz_inits(Y, F, NULL);
	mpz_import(Y, nlimbs, -1, 8, 0, 0, y);
	free(y);
	if (f != 0)
	{
		mpz_set_si(F, (long)f);
		mpz_mul_2exp(F, F, (mp_bitcnt_t)nbits);
		mpz_add(Y, Y, F);
	}
	mpz_mod(Y, Y, o->N);
	const size_t sz = mpz_size(Y);
	long ret = -1;
	if (sz <= cap) { for (size_t i = 0; i < sz; ++i) out[i] = mpz_getlimbn(Y, (mp_size_t)i); ret = (long)sz; }
	mpz_clears(Y, F, NULL);
	return ret;
}

void or_get_factor(void * h, uint64_t * out, size_t cap, size_t * count)
{
	oracle * o = (oracle *)h;
	const size_t sz = mpz_size(o->factor);
	*count = 0;
	if (sz > cap) return;
	for (size_t i = 0; i < sz; ++i) out[i] = mpz_getlimbn(o->factor, (mp_size_t)i);
	*count = sz;
}

void or_info(void * h, int * K, int * pck, int * ln, int * lbase)
{
	oracle * o = (oracle *)h; *K = o->K; *pck = o->pck; *ln = o->ln; *lbase = o->lbase;
}
