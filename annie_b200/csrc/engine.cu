// Host engine of the modular-squaring transform and its C ABI
// (include/annie_b200.h).
//
// The engine owns all device memory of one transform, drives the two NTT
// passes of kernels.cu in the Montgomery-McLaughlin-Gallot-Woltman (MMGW)
// sequence of the reference (src/transformGPU.h:523-568) and converts
// integers to and from the RNS register layout on the host
// (src/transformGPU.h:323-445).
#include <cstdint>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <stdexcept>
#include <algorithm>
#include <atomic>
#include <map>
#include <memory>
#include <thread>
#include <mutex>
#include <tuple>
#include <cuda_runtime.h>

#include "gmp.h"
#include "kernels.h"
#include "../../include/annie_b200.h"
#include "../../include/annie_b200_batch.h"

using namespace ab;

namespace
{
thread_local std::string g_last_error;

struct ab_error : std::runtime_error
{
	int code;
	ab_error(int c, const std::string & m) : std::runtime_error(m), code(c) {}
};

#define CK(call) do { const cudaError_t e_ = (call); if (e_ != cudaSuccess) throw ab_error(AB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); } while (0)

// ------------------------------------------------------------ host Z/pZ
// The 14 primes of the reference and their primitive roots
// (src/transformGPU.h:79-89): the parameter rule and the register words of
// the reference's normal form use them.
const u32 PRIMES[14] = {
	(125u << 25) + 1, (243u << 24) + 1, (235u << 24) + 1, (29u << 27) + 1,
	(13u << 28) + 1, (193u << 24) + 1, (3u << 30) + 1, (43u << 26) + 1,
	(171u << 24) + 1, (81u << 25) + 1, (157u << 24) + 1, (151u << 24) + 1,
	(37u << 26) + 1, (17u << 27) + 1 };

// The transform primes: p < 2^30, p = c 2^23 + 1 (roots of unity of order
// 2^23 cover both domains up to n = 2^22), largest first, with a generator of
// each multiplicative group.  A class with K reference primes uses the first
// K + 1: their product exceeds the reference's (2^89.4 > 2^63.9 for K = 2,
// 2^118.8 > 2^95.8, 2^148.1 > 2^127.6, 2^177.3 > 2^159.3 for K = 5).
const u32 TPRIMES[AB_MAXKP] = { 119u * (1u << 23) + 1, 107u * (1u << 23) + 1, 105u * (1u << 23) + 1,
                                90u * (1u << 23) + 1, 77u * (1u << 23) + 1, 71u * (1u << 23) + 1 };
const u32 TGEN[AB_MAXKP] = { 3, 3, 26, 11, 3, 3 };

// Montgomery arithmetic mod a reference prime (canonical values)
struct HostZp
{
	u32 p, q, one, rsq;
	explicit HostZp(u32 pp) : p(pp)
	{
		q = 1; for (int i = 0; i < 6; ++i) q *= 2 - p * q;      // p^-1 mod 2^32 (Newton)
		one = (u32)(((u64)1 << 32) % p);
		rsq = (u32)(((u64)one * one) % p);
	}
	u32 sub(u32 a, u32 b) const { return a - b + ((a < b) ? p : 0); }
	u32 mul(u32 a, u32 b) const
	{
		const u64 t = (u64)a * b; const u32 m = (u32)t * q;
		return sub((u32)(t >> 32), (u32)(((u64)m * p) >> 32));
	}
	u32 to_mont(u32 a) const { return mul(a % p, rsq); }
	u32 pow(u32 x, u32 e) const { u32 r = one; while (e) { if (e & 1) r = mul(r, x); x = mul(x, x); e >>= 1; } return r; }
	u32 inv(u32 x) const { return pow(x, p - 2); }
};

// Plain arithmetic mod a transform prime
struct TZp
{
	u32 p;
	explicit TZp(u32 pp) : p(pp) {}
	u32 mul(u32 a, u32 b) const { return (u32)(((u64)a * b) % p); }
	u32 pow(u32 x, u64 e) const { u32 r = 1; while (e) { if (e & 1) r = mul(r, x); x = mul(x, x); e >>= 1; } return r; }
	u32 inv(u32 x) const { return pow(x, p - 2); }
	u32 shoup(u32 w) const { return (u32)(((u64)w << 32) / p); }
};

size_t bitrev(size_t i, size_t n)
{
	size_t r = 0;
	for (size_t k = n, j = i; k > 1; k /= 2, j /= 2) r = (2 * r) | (j % 2);
	return r;
}

// Twiddles of transform prime k for length 2^ln at the reference's positions
// s + bitrev(j, s), s = n/4 .. 1 (transformGPU.h:117-160; position 0 unused).
// Domain R (x^n - 1): w = rho_s^j with rho_s a primitive 2s-th root of unity;
// the inverse levels use -rho_s^-j.  Domain Q (x^n + 1), twisted:
// w = psi_s rho_s^j with psi_s a primitive 4s-th root (psi_s^2 = rho_s), and
// -w_j^-1 = w_{s-1-j}, the forward twiddle at the mirrored position.
// Outputs, as Shoup pairs (w, floor(w 2^32 / p)): the row tables (w, and wi
// for domain R only), and the column tables (the first COLTW positions),
// forward cf and inverse ci (both domains).
void make_twiddles(uint2 * w, uint2 * wi, uint2 * cf, uint2 * ci, int ln, int k, bool domain_q)
{
	const TZp z(TPRIMES[k]);
	const size_t n = (size_t)1 << ln, h = n / 2, nc = std::min<size_t>(h, COLTW);
	auto root = [&](int l) { return z.pow(TGEN[k], (z.p - 1) >> l); };     // primitive 2^l-th root
	std::vector<u32> fw(h, 0), iw(h, 0);                  // plain values
	int l = ln - 1;                                       // rho of the level s = n/4 has order 2^(ln-1)
	for (size_t s = n / 4; s >= 1; s /= 2, --l)
	{
		const u32 rho = root(l), rhoi = z.inv(rho);
		u32 t = domain_q ? root(l + 1) : 1u, ti = 1u;
		for (size_t j = 0; j < s; ++j)
		{
			const size_t jr = bitrev(j, s);
			fw[s + jr] = t;
			iw[s + jr] = (z.p - ti) % z.p;
			t = z.mul(t, rho); ti = z.mul(ti, rhoi);
		}
	}
	if (domain_q)
		for (size_t s = n / 4; s >= 1; s /= 2)
			for (size_t i = s; i < 2 * s; ++i) iw[i] = fw[3 * s - 1 - i];     // -w^-1 (same values as above)
	for (size_t i = 0; i < h; ++i)
	{
		w[i] = make_uint2(fw[i], z.shoup(fw[i]));
		if (wi) wi[i] = make_uint2(iw[i], z.shoup(iw[i]));
	}
	for (size_t i = 0; i < COLTW; ++i)
	{
		const u32 a = (i < nc) ? fw[i] : 0u, bb = (i < nc) ? iw[i] : 0u;
		cf[i] = make_uint2(a, z.shoup(a));
		ci[i] = make_uint2(bb, z.shoup(bb));
	}
}

size_t get_s(size_t K) { int s = -1; for (size_t k = K - 1; k != 0; k /= 2) ++s; return (size_t)1 << s; }

// Parameter rule of the reference factory (transformGPU.h:798-850): for
// K = 2..5 primes with packing get_s(K), the largest digit size that keeps
// ln + 2 pck lbase < log2(prod P / 2a); keep the K with the smallest K n ln.
void get_n_base(int & rln, int & rlbase, int pck, double log2_16aN, double log2_p_2a)
{
	for (int lbase = 31; lbase >= 2; --lbase)
	{
		int ln = 4; while (double(lbase * pck) * (1 << ln) < log2_16aN) ++ln;
		const int log2_base = lbase * pck;
		if (ln + 2 * log2_base < log2_p_2a) { rln = ln; rlbase = lbase; break; }
	}
}

ab_params select_params(const mpz_t N, int32_t a)
{
	long e_n; const double m_n = mpz_get_d_2exp(&e_n, N);
	const double log2_16aN = std::log2(16.0 * a) + std::log2(m_n) + e_n;
	double l = std::log2(double(PRIMES[0])) - std::log2(2.0 * a);
	uint64_t c_min = uint64_t(-1); size_t K_min = 0;
	for (size_t K = 2; K < 6; ++K)
	{
		l += std::log2(double(PRIMES[K - 1]));
		int ln = 0, lbase = 0; get_n_base(ln, lbase, (int)get_s(K), log2_16aN, l);
		const uint64_t c = K * uint64_t(1u << ln) * uint64_t(ln);
		if (c < c_min) { c_min = c; K_min = K; }
	}
	l = std::log2(double(PRIMES[0])) - std::log2(2.0 * a);
	for (size_t k = 1; k < K_min; ++k) l += std::log2(double(PRIMES[k]));
	ab_params p; p.K = (int)K_min; p.pck = (int)get_s(K_min); p.ln = 0; p.lbase = 0;
	get_n_base(p.ln, p.lbase, p.pck, log2_16aN, l);
	return p;
}

void mpz_from_limbs(mpz_t z, const uint64_t * limbs, size_t n) { mpz_import(z, n, -1, 8, 0, 0, limbs); }

// 0: ok, else R = base^(pck n) - 1 shares a factor with N (stored in factor)
bool compute_R_Ninv(const mpz_t N, const ab_params & p, mpz_t R, mpz_t Ninv, mpz_t factor)
{
	mpz_set_ui(R, 1);
	mpz_mul_2exp(R, R, (mp_bitcnt_t)p.pck * (mp_bitcnt_t)p.lbase << p.ln);
	mpz_sub_ui(R, R, 1);
	if (mpz_invert(Ninv, N, R) == 0) { mpz_gcd(factor, N, R); return false; }
	return true;
}
} // namespace

// ============================================================ allocation-free squaring
// Work buffers of ab_square_mul_noalloc: five regions of AB_NOALLOC_MAX_WORDS
// words (10 MiB; four NTT-form buffers, then T_Q and the register's exact
// values) and a flag word, in a static device array that
// every GPU loading this library holds until the process exits.  Host code
// cannot use the symbol as an address: the device address is fetched with
// cudaGetSymbolAddress, with that device current, once per device -- when a
// transform or a batch is created there, so that the entry point itself only
// queues kernels.
#define AB_NOALLOC_MAX_WORDS (1u << 19)
#define AB_NOALLOC_MAX_DEVICES 64
static __device__ __align__(256) u32 g_noalloc_scratch[5 * AB_NOALLOC_MAX_WORDS + 64];

namespace
{
std::mutex g_noalloc_mu;
u32 * g_noalloc_addr[AB_NOALLOC_MAX_DEVICES] = {};

u32 * noalloc_scratch(int device)
{
	if (device < 0 || device >= AB_NOALLOC_MAX_DEVICES) throw ab_error(AB_E_ARG, "device index out of range");
	std::lock_guard<std::mutex> lock(g_noalloc_mu);
	if (g_noalloc_addr[device] == nullptr)
	{
		int prev = 0;
		CK(cudaGetDevice(&prev));
		CK(cudaSetDevice(device));
		void * p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		cudaSetDevice(prev);
		if (e != cudaSuccess) throw ab_error(AB_E_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
		g_noalloc_addr[device] = static_cast<u32 *>(p);
	}
	return g_noalloc_addr[device];
}
}

// ============================================================ the engine
struct ab_transform
{
	// Device buffers.  Normal form (AB_NW = 3 planes of n words, exact
	// coefficient values): the registers, the MMGW one, T_Q, TMP, the
	// Gerbicz-Li snapshot.  NTT form (KP planes): the four partly transformed
	// work buffers, the transforms of N (domain Q) and N^-1 (domain R), two
	// transformed multiplicands.  Shared by the slots of a batch: XW (the
	// reference's register words, K planes, for conversions), the row twiddle
	// tables (KP n/2 words each) and the column twiddle tables (WC: domains R,
	// Q x forward, inverse x KP primes x COLTW Shoup pairs).
	enum Buf { REG0 = 0, REG1, REG2, ONE, TQ, TMP, SNAP, AQ0, AQ1, AR0, AR1, NQ, NIR, OPQ, OPR, NSLOT = OPR + 1,
	           XW = NSLOT, WR, WRI, WQ, WC, NBUF };
	static bool normal_buf(int i) { return i <= SNAP; }

	int device = 0;
	cudaStream_t st = nullptr;
	cudaStream_t st2 = nullptr;          // Q-domain chain, joined before the carry-sub
	cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_fork = nullptr, ev_q = nullptr;
	bool overlap = true;                 // run the Q chain on st2 (off for per-launch profiling)
	bool split = false;                  // without overlap: still one launch per domain
	ab_params prm{};
	int KP = 0;                          // transform primes
	size_t n = 0;
	Geometry geo{};
	TConst tc{};
	RefConst rc{};
	bool failed = false;
	mpz_t N, factor;
	u32 * dmem = nullptr;
	u32 * d_flag = nullptr;              // import error flag (device word)
	bool prefwd = false;     // AR0 (and AQ0 unless q_pending) hold the first forward levels of REG0
	bool q_pending = false;  // AQ0 is still to be computed from REG0, at the head of the Q chain
	std::vector<u32> host;
	uint64_t launches = 0;   // kernels launched by this handle
	std::vector<cudaEvent_t> prof;   // non-empty: record an event before every launch
	size_t prof_used = 0;
	void * flush_buf = nullptr;

	u32 * bufp[NBUF] = {};   // device buffers (a batch slot view points into its batch)
	u32 * noalloc = nullptr; // device address of the static scratch of ab_square_mul_noalloc on this device
	bool view = false;       // true: memory and streams belong to a batch

	// runs of squarings replayed from a captured CUDA graph: GRAPH_STEPS
	// squarings whose multipliers are read from d_mult, uploaded from
	// page-locked staging (two buffers, each reused once its upload is done)
	static const int GRAPH_STEPS = 64;
	cudaGraphExec_t gexec = nullptr;
	uint64_t graph_kernels = 0;          // kernel nodes in gexec
	u32 * d_mult = nullptr;
	u32 * h_mult[2] = {};
	cudaEvent_t mult_done[2] = {};
	int mult_i = 0;

	u32 * b(int i) const { return bufp[i]; }
	static size_t words_of(int i, int K, size_t n)
	{
		if (i == XW) return (size_t)K * n;
		if (i == WR || i == WRI || i == WQ) return (size_t)(K + 1) * n;        // n/2 pairs per prime
		if (i == WC) return (size_t)4 * (K + 1) * COLTW * 2;
		return (i < NSLOT && normal_buf(i)) ? (size_t)AB_NW * n : (size_t)(K + 1) * n;
	}
	size_t words_of(int i) const { return words_of(i, prm.K, n); }

	ab_transform() { mpz_inits(N, factor, nullptr); }
	ab_transform(const ab_transform &) = delete;
	ab_transform & operator=(const ab_transform &) = delete;

	~ab_transform()
	{
		if (view) { mpz_clears(N, factor, nullptr); return; }
		for (cudaEvent_t e : prof) cudaEventDestroy(e);
		if (gexec) cudaGraphExecDestroy(gexec);
		if (d_mult) cudaFree(d_mult);
		for (int i = 0; i < 2; ++i) { if (h_mult[i]) cudaFreeHost(h_mult[i]); if (mult_done[i]) cudaEventDestroy(mult_done[i]); }
		if (flush_buf) cudaFree(flush_buf);
		if (dmem) cudaFree(dmem);
		if (ev0) cudaEventDestroy(ev0);
		if (ev1) cudaEventDestroy(ev1);
		if (ev_fork) cudaEventDestroy(ev_fork);
		if (ev_q) cudaEventDestroy(ev_q);
		if (st2) cudaStreamDestroy(st2);
		if (st) cudaStreamDestroy(st);
		mpz_clears(N, factor, nullptr);
	}

	// Constants of the transform primes (TConst) and of the reference primes
	// (RefConst) for the class (K, pck, ln) and digit size lbase.
	static void build_consts(const ab_params & prm, const Geometry & geo, TConst & tc, RefConst & rc)
	{
		const int K = prm.K, KP = K + 1, L = K;
		const size_t n = (size_t)1 << prm.ln;
		std::memset(&tc, 0, sizeof(tc));
		tc.K = K; tc.KP = KP; tc.pck = prm.pck; tc.lbase = prm.lbase; tc.ln = prm.ln;
		tc.n = (u32)n;
		apply_geometry(tc, geo);
		mpz_t M, Mk, t, mod; mpz_inits(M, Mk, t, mod, nullptr);
		mpz_set_ui(M, 1);
		for (int k = 0; k < KP; ++k) mpz_mul_ui(M, M, TPRIMES[k]);
		mpz_set_ui(mod, 1); mpz_mul_2exp(mod, mod, (mp_bitcnt_t)32 * L);
		auto limbs = [&](const mpz_t v, u32 * out) {
			mpz_fdiv_r(t, v, mod);
			for (int j = 0; j < L; ++j) { out[j] = (u32)mpz_get_ui(t); mpz_fdiv_q_2exp(t, t, 32); }
		};
		for (int k = 0; k < KP; ++k)
		{
			const TZp z(TPRIMES[k]);
			const u32 p = z.p;
			tc.p[k] = p;
			u32 pinv = 1; for (int i = 0; i < 6; ++i) pinv *= 2 - p * pinv;
			tc.pinv[k] = pinv;
			tc.one_s[k] = z.shoup(1);
			tc.c32[k] = (u32)(((u64)1 << 32) % p); tc.c32s[k] = z.shoup(tc.c32[k]);
			tc.c64[k] = z.mul(tc.c32[k], tc.c32[k]); tc.c64s[k] = z.shoup(tc.c64[k]);
			const u32 p95 = z.mul(tc.c64[k], (u32)(((u64)1 << 31) % p));
			tc.k95[k] = (p - p95) % p;
			mpz_divexact_ui(Mk, M, p);
			const u32 mk_mod_p = (u32)mpz_fdiv_ui(Mk, p);
			// (2/n) 2^32 (M/p)^-1: undoes the n/2 of the inverse levels and the
			// 2^-32 of the Montgomery pointwise product, and weights the CRT
			tc.crt[k] = z.mul(z.mul(z.inv((u32)((n / 2) % p)), tc.c32[k]), z.inv(mk_mod_p));
			tc.crts[k] = z.shoup(tc.crt[k]);
			tc.fl[k] = (u32)(((u64)1 << 60) / p);
			limbs(Mk, tc.mk[k]);
		}
		mpz_neg(t, M);
		limbs(t, tc.negm);
		mpz_clears(M, Mk, t, mod, nullptr);

		std::memset(&rc, 0, sizeof(rc));
		rc.K = K;
		for (int k = 0; k < K; ++k)
		{
			const HostZp z(PRIMES[k]);
			rc.p[k] = z.p; rc.q[k] = z.q;
			rc.r2[k] = (u32)((((u64)z.one) * z.one) % z.p);          // 2^64 mod p
			for (int j = k + 1; j < K; ++j)
			{
				rc.gm[k][j] = z.inv(z.to_mont(PRIMES[j] % z.p));       // Montgomery form of P_j^-1
				rc.gmq[k][j] = rc.gm[k][j] * z.q;
			}
		}
	}

	// integer -> exact coefficient values: pck digits of lbase bits per
	// coefficient (transformGPU.h:323-360), three limb planes
	void encode(const mpz_t x, u32 * out) const
	{
		const size_t nl = mpz_size(x);
		const u64 * xl = (const u64 *)mpz_limbs_read(x);
		const int lb = prm.lbase;
		auto read_bits = [&](size_t bit) -> u32 {
			const size_t li = bit / 64; const int sh = (int)(bit % 64);
			const u64 lo = (li < nl) ? xl[li] : 0, hi = (li + 1 < nl) ? xl[li + 1] : 0;
			u64 r = lo >> sh; if (sh != 0) r |= hi << (64 - sh);
			return (u32)r & ((1u << lb) - 1);
		};
		size_t bit = 0;
		for (size_t i = 0; i < n; ++i)
		{
			unsigned __int128 d = 0;
			u32 dg[4];
			for (int l = 0; l < prm.pck; ++l) { dg[l] = read_bits(bit); bit += (size_t)lb; }
			for (int l = prm.pck - 1; l >= 0; --l) d = (d << lb) | dg[l];
			out[i] = (u32)d; out[n + i] = (u32)(d >> 32); out[2 * n + i] = (u32)(d >> 64);
		}
	}

	// exact coefficient values -> integer sum_i v_i 2^(pck lbase i), then mod N
	// (transformGPU.h:362-445 does the same from the residues)
	void decode(const u32 * planes, mpz_t y) const
	{
		const int w = prm.pck * prm.lbase;
		const size_t nbits = (size_t)w * n, nlimbs = nbits / 64 + 2;
		std::vector<u64> out(nlimbs, 0);
		__int128 f = 0; size_t bit = 0;
		auto put = [&](u64 r, int cnt) {
			const size_t li = bit / 64; const int sh = (int)(bit % 64);
			out[li] |= r << sh; if (sh != 0 && sh + cnt > 64) out[li + 1] |= r >> (64 - sh);
			bit += (size_t)cnt;
		};
		for (size_t i = 0; i < n; ++i)
		{
			const unsigned __int128 u = (unsigned __int128)planes[i] | ((unsigned __int128)planes[n + i] << 32) |
			                            ((unsigned __int128)planes[2 * n + i] << 64);
			f += (__int128)(u << 32) >> 32;           // sign-extended 96-bit value
			for (int left = w; left > 0;)
			{
				const int cnt = std::min(left, 32);
				put((u64)(f & ((((__int128)1) << cnt) - 1)), cnt);
				f >>= cnt; left -= cnt;
			}
		}
		mpz_import(y, nlimbs, -1, 8, 0, 0, out.data());
		if (f != 0)
		{
			mpz_t F; mpz_init(F);
			mpz_set_si(F, (long)f);
			mpz_mul_2exp(F, F, (mp_bitcnt_t)nbits);
			mpz_add(y, y, F);
			mpz_clear(F);
		}
		mpz_mod(y, y, N);
	}

	// ---------------------------------------------------------- pass helpers
	void mark()
	{
		if (prof_used < prof.size()) CK(cudaEventRecord(prof[prof_used++], st));
	}
	// a row pass, with the mid levels before and after it above 2^20
	void rows(const RowJob & j0, const RowJob * j1 = nullptr, cudaStream_t s = nullptr)
	{
		RowJobs js; js.j[0] = j0; js.j[1] = j1 ? *j1 : j0;
		const int nj = j1 ? 2 : 1;
		if (s == nullptr) { mark(); s = st; }
		if (geo.G > 0) { CK(launch_midpass(geo, tc, js, nj, s, 1, false)); ++launches; }
		CK(launch_rowpass(geo, tc, js, nj, s));
		++launches;
		if (geo.G > 0 && j0.mode != ROW_FWD_ONLY) { CK(launch_midpass(geo, tc, js, nj, s, 1, true)); ++launches; }
	}
	void cols(const ColJob & j0, const ColJob * j1 = nullptr, cudaStream_t s = nullptr)
	{
		ColJobs js; js.j[0] = j0; js.j[1] = j1 ? *j1 : j0;
		if (s == nullptr) { mark(); s = st; }
		CK(launch_colpass(geo, tc, js, j1 ? 2 : 1, s));
		++launches;
	}
	// twiddles of a domain (q: Q, else R): row tables, and the column tables
	// (forward, inverse) of WC
	const uint2 * wf(bool q) const { return reinterpret_cast<const uint2 *>(b(q ? WQ : WR)); }
	const uint2 * wv(bool q) const { return q ? nullptr : reinterpret_cast<const uint2 *>(b(WRI)); }
	const uint2 * wc(bool q, bool inverse) const { return reinterpret_cast<const uint2 *>(b(WC)) + ((q ? 2 : 0) + (inverse ? 1 : 0)) * KP * COLTW; }
	RowJob rj(u32 * x, int mode, bool q, const u32 * xp = nullptr) const
	{
		RowJob j; std::memset(&j, 0, sizeof(j)); j.x = x; j.xp = xp; j.w = wf(q); j.wi = wv(q); j.mode = mode; return j;
	}
	ColJob cj_norm(const u32 * in) const
	{
		ColJob j; std::memset(&j, 0, sizeof(j)); j.in = in; j.transformed = 0; j.a = 1; return j;
	}
	ColJob cj_tr(const u32 * in, bool q, u32 a, const u32 * sub, int lower) const
	{
		ColJob j; std::memset(&j, 0, sizeof(j));
		j.in = in; j.transformed = 1; j.wi_in = wc(q, true); j.a = a; j.nega = q ? 1 : 0; j.sub = sub; j.lower = lower;
		return j;
	}
	void set_fwd(ColJob & j, u32 * q_out, u32 * r_out) const
	{
		j.out_fwd[0] = q_out; j.w_out[0] = q_out ? wc(true, false) : nullptr;
		j.out_fwd[1] = r_out; j.w_out[1] = r_out ? wc(false, false) : nullptr;
	}

	// full forward transform of a normal-form register in one or two domains
	void full_forward(const u32 * src, u32 * dq, u32 * dr)
	{
		ColJob j = cj_norm(src); set_fwd(j, dq, dr); cols(j);
		if (dq && dr) { RowJob a = rj(dq, ROW_FWD_ONLY, true), c = rj(dr, ROW_FWD_ONLY, false); rows(a, &c); }
		else if (dq) rows(rj(dq, ROW_FWD_ONLY, true));
		else rows(rj(dr, ROW_FWD_ONLY, false));
	}

	// reduceMMGW tail (transformGPU.h:523-538): m' = T_R Ninv mod R, +2,
	// r' = m' N - T_Q mod Q.  AR1 holds the first forward levels of T_R.
	// With the Q chain on its own stream, the carry-sub leaves only the R-domain
	// levels (the next squaring's critical path starts there); the Q chain
	// starts by computing its own from the new Reg0 (q_pending).
	void reduce_tail(const u32 * tq, u32 * out, bool want_prefwd, bool join_q = false)
	{
		rows(rj(b(AR1), ROW_MUL, false, b(NIR)));
		ColJob j1 = cj_tr(b(AR1), false, 1, nullptr, LOWER_R_ADD2); set_fwd(j1, b(AQ1), nullptr); cols(j1);
		rows(rj(b(AQ1), ROW_MUL, true, b(NQ)));
		if (join_q) CK(cudaStreamWaitEvent(st, ev_q, 0));
		ColJob j2 = cj_tr(b(AQ1), true, 1, tq, LOWER_Q); j2.out_norm = out;
		const bool q_chain = overlap || split;   // the Q chain has launches of its own
		if (want_prefwd) set_fwd(j2, q_chain ? nullptr : b(AQ0), b(AR0));
		cols(j2);
		q_pending = want_prefwd && q_chain;
	}

	// First product of squareMMGW / mulMMGW (transformGPU.h:540-568):
	// T_Q = carry(x y mod Q) into TQ and the first forward levels of
	// carry(x y mod R) into AR1.  AQ0/AR0 hold the first forward levels of x;
	// xq/xr the full forward images of y (nullptr: y = x, square).  With
	// overlap, the Q chain runs on st2 (T_Q is only needed by the final
	// carry-sub) and reduce_tail joins it.  A non-null `mult` is a device word
	// read in place of `a` (graph replays).
	void first_product(u32 a, const u32 * xq, const u32 * xr, const u32 * mult = nullptr, bool q_from_reg0 = false)
	{
		RowJob rq = rj(b(AQ0), xq ? ROW_MUL : ROW_SQUARE, true, xq), rr = rj(b(AR0), xr ? ROW_MUL : ROW_SQUARE, false, xr);
		ColJob jq = cj_tr(b(AQ0), true, a, nullptr, LOWER_NONE); jq.out_norm = b(TQ); jq.mult = mult;
		ColJob jr = cj_tr(b(AR0), false, a, nullptr, LOWER_NONE); set_fwd(jr, nullptr, b(AR1)); jr.mult = mult;
		if (overlap)
		{
			CK(cudaEventRecord(ev_fork, st));
			CK(cudaStreamWaitEvent(st2, ev_fork, 0));
			if (q_from_reg0) { ColJob jf = cj_norm(b(REG0)); set_fwd(jf, b(AQ0), nullptr); cols(jf, nullptr, st2); }
			rows(rq, nullptr, st2);
			cols(jq, nullptr, st2);
			CK(cudaEventRecord(ev_q, st2));
			rows(rr);
			cols(jr);
		}
		else
		{
			if (q_from_reg0) { ColJob jf = cj_norm(b(REG0)); set_fwd(jf, b(AQ0), nullptr); cols(jf); }
			if (split)
			{
				// the launches of the overlapped schedule, in order on one stream
				rows(rq); cols(jq); rows(rr); cols(jr);
			}
			else
			{
				rows(rq, &rr);
				cols(jq, &jr);
			}
		}
	}

	void prefwd_reg0()
	{
		if (!prefwd) { ColJob j = cj_norm(b(REG0)); set_fwd(j, b(AQ0), b(AR0)); cols(j); q_pending = false; }
	}

	// squareMMGW (transformGPU.h:556-568)
	void square_mul(u32 a)
	{
		prefwd_reg0();
		first_product(a, nullptr, nullptr, nullptr, q_pending);
		reduce_tail(b(TQ), b(REG0), true, overlap);
		prefwd = true;
	}

	// GRAPH_STEPS squarings with multipliers mults[0..GRAPH_STEPS) from the graph
	void square_mul_graph(const u32 * mults)
	{
		const int G = GRAPH_STEPS;
		if (d_mult == nullptr)
		{
			CK(cudaMalloc(&d_mult, G * sizeof(u32)));
			for (int i = 0; i < 2; ++i)
			{
				CK(cudaMallocHost(&h_mult[i], G * sizeof(u32)));
				CK(cudaEventCreateWithFlags(&mult_done[i], cudaEventDisableTiming));
				CK(cudaEventRecord(mult_done[i], st));
			}
		}
		if (gexec == nullptr)
		{
			RowJobs rjs{}; ColJobs cjs{};
			CK(launch_rowpass(geo, tc, rjs, 1, st, 0));     // kernel attributes, outside the capture
			CK(launch_colpass(geo, tc, cjs, 1, st, 0));
			const uint64_t l0 = launches;
			cudaGraph_t g = nullptr;
			CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
			try
			{
				for (int s = 0; s < G; ++s)
				{
					first_product(1, nullptr, nullptr, d_mult + s, overlap);
					reduce_tail(b(TQ), b(REG0), true, overlap);
				}
			}
			catch (...) { cudaStreamEndCapture(st, &g); if (g) cudaGraphDestroy(g); launches = l0; throw; }
			CK(cudaStreamEndCapture(st, &g));
			graph_kernels = launches - l0;       // counted by rows()/cols() while recording
			launches = l0;
			const cudaError_t ei = cudaGraphInstantiate(&gexec, g, 0);
			cudaGraphDestroy(g);
			CK(ei);
		}
		prefwd_reg0();                           // AR0 (and AQ0, recomputed by the graph's first step)
		const int hi = mult_i;
		CK(cudaEventSynchronize(mult_done[hi]));
		std::memcpy(h_mult[hi], mults, G * sizeof(u32));
		CK(cudaMemcpyAsync(d_mult, h_mult[hi], G * sizeof(u32), cudaMemcpyHostToDevice, st));
		CK(cudaEventRecord(mult_done[hi], st));
		mult_i ^= 1;
		CK(cudaGraphLaunch(gexec, st));
		launches += graph_kernels;
		prefwd = true;
		q_pending = overlap;                     // as the graph's last step left it
	}

	// the split and the launch constants that describe it, always together
	void use_geometry(const Geometry & g)
	{
		geo = g;
		apply_geometry(tc, g);
	}

	// row/column split of the transform (the register layouts do not depend on it)
	void set_geometry(int lb)
	{
		Geometry g;
		if (!make_geometry(prm.ln, lb, g)) throw ab_error(AB_E_ARG, "geometry not available for this length");
		CK(cudaStreamSynchronize(st));
		use_geometry(g);
		prefwd = false;                          // AQ0/AR0 hold levels of the old split
		if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
	}

	// mulMMGW (transformGPU.h:540-554)
	void mul(int dst, int src)
	{
		full_forward(b(src), b(OPQ), b(OPR));
		{ ColJob j = cj_norm(b(dst)); set_fwd(j, b(AQ0), b(AR0)); cols(j); }
		prefwd = false;
		first_product(1, b(OPQ), b(OPR));
		reduce_tail(b(TQ), b(dst), dst == REG0, overlap);
		prefwd = (dst == REG0);
	}

	// conversion out of MMGW form into TMP (transformGPU.h:576-586)
	void reduce_copy(int src)
	{
		ColJob j = cj_norm(b(src)); set_fwd(j, nullptr, b(AR1)); cols(j);
		reduce_tail(b(src), b(TMP), false);
	}

	void copy(int dst, int src)
	{
		if (dst == src) return;
		CK(cudaMemcpyAsync(b(dst), b(src), words_of(dst) * 4, cudaMemcpyDeviceToDevice, st));
		if (dst == REG0) prefwd = false;
	}

	void upload(int buf, const u32 * src)
	{
		CK(cudaMemcpyAsync(b(buf), src, words_of(buf) * 4, cudaMemcpyHostToDevice, st));
		CK(cudaStreamSynchronize(st));
	}
	void download(int buf, u32 * dst, size_t words)
	{
		CK(cudaMemcpyAsync(dst, b(buf), words * 4, cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
	}

	// the reference's register words (K planes) of a normal-form buffer, into XW
	void export_words(int buf)
	{
		CK(launch_export(rc, b(buf), b(XW), (u32)n, st));
		++launches;
	}
	// XW (the reference's register words) into a normal-form buffer; returns
	// false when they are not a normal-form register
	bool import_words(int buf)
	{
		CK(cudaMemsetAsync(d_flag, 0, sizeof(u32), st));
		CK(launch_import(rc, b(XW), b(buf), (u32)n, d_flag, st));
		++launches;
		u32 bad = 0;
		CK(cudaMemcpyAsync(&bad, d_flag, sizeof(u32), cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		if (buf == REG0) prefwd = false;
		return bad == 0;
	}

	void get(int src, mpz_t z)
	{
		reduce_copy(src);
		host.resize((size_t)AB_NW * n);
		download(TMP, host.data(), (size_t)AB_NW * n);
		decode(host.data(), z);
	}

	// host part of the set-up: parameters, geometry, R, N^-1 mod R, constants,
	// and the exact values of N, N^-1 and the MMGW form of 1
	struct Prepared
	{
		std::vector<u32> wN, wNinv, wOne;
	};

	void prepare(const mpz_t Nin, int32_t a, const ab_params * forced, Prepared & pp)
	{
		mpz_set(N, Nin);
		prm = forced ? *forced : select_params(N, a);
		if (prm.K < 2 || prm.K > 5 || (size_t)prm.pck != get_s((size_t)prm.K) || prm.lbase < 2 || prm.lbase > 31 ||
		    prm.pck * prm.lbase > 80)
			throw ab_error(AB_E_ARG, "invalid transform parameters");
		if (!make_geometry(prm.ln, 0, geo)) throw ab_error(AB_E_UNSUPPORTED, "NTT length 2^" + std::to_string(prm.ln) + " is not supported (6 <= ln <= 22)");
		n = (size_t)1 << prm.ln;
		KP = prm.K + 1;
		mpz_t R, Ninv; mpz_inits(R, Ninv, nullptr);
		if (!compute_R_Ninv(N, prm, R, Ninv, factor)) { failed = true; mpz_clears(R, Ninv, nullptr); return; }
		build_consts(prm, geo, tc, rc);
		const size_t words = (size_t)AB_NW * n;
		pp.wN.resize(words); pp.wNinv.resize(words); pp.wOne.resize(words);
		encode(N, pp.wN.data());
		encode(Ninv, pp.wNinv.data());
		// MMGW form of 1 is R/2 mod N (transformGPU.h:743-747)
		mpz_mod(Ninv, R, N);
		if (mpz_odd_p(Ninv)) mpz_add(Ninv, Ninv, N);
		mpz_fdiv_q_2exp(Ninv, Ninv, 1);
		encode(Ninv, pp.wOne.data());
		mpz_clears(R, Ninv, nullptr);
	}

	// device part: forward transforms of N (domain Q) and N^-1 (domain R), and 1
	void setup_device(const Prepared & pp)
	{
		upload(TMP, pp.wN.data());
		full_forward(b(TMP), b(NQ), nullptr);
		upload(TMP, pp.wNinv.data());
		full_forward(b(TMP), nullptr, b(NIR));
		upload(ONE, pp.wOne.data());
		CK(cudaStreamSynchronize(st));
	}

	// twiddle tables of the class (host): row tables WR, WRI, WQ (KP n/2 pairs
	// each) and the column tables WC
	static void twiddle_tables(const ab_params & prm, std::vector<uint2> & wr, std::vector<uint2> & wri, std::vector<uint2> & wq,
	                           std::vector<uint2> & wc)
	{
		const size_t h = (size_t)1 << (prm.ln - 1);
		const int KP = prm.K + 1;
		wr.assign(KP * h, make_uint2(0, 0)); wri.assign(KP * h, make_uint2(0, 0)); wq.assign(KP * h, make_uint2(0, 0));
		wc.assign((size_t)4 * KP * COLTW, make_uint2(0, 0));
		for (int k = 0; k < KP; ++k)
		{
			uint2 * const c = wc.data();
			make_twiddles(&wr[k * h], &wri[k * h], c + (0 * KP + k) * COLTW, c + (1 * KP + k) * COLTW, prm.ln, k, false);
			make_twiddles(&wq[k * h], nullptr, c + (2 * KP + k) * COLTW, c + (3 * KP + k) * COLTW, prm.ln, k, true);
		}
	}

	void upload_twiddles()
	{
		std::vector<uint2> wr, wri, wq, wcv;
		twiddle_tables(prm, wr, wri, wq, wcv);
		CK(cudaMemcpyAsync(b(WR), wr.data(), wr.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(b(WRI), wri.data(), wri.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(b(WQ), wq.data(), wq.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(b(WC), wcv.data(), wcv.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
		CK(cudaStreamSynchronize(st));
	}

	void init(const mpz_t Nin, int32_t a, int dev, const ab_params * forced)
	{
		device = dev;
		Prepared pp;
		prepare(Nin, a, forced, pp);
		if (failed) return;

		CK(cudaSetDevice(device));
		noalloc = noalloc_scratch(device);
		CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
		CK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
		CK(cudaEventCreate(&ev0)); CK(cudaEventCreate(&ev1));
		CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
		CK(cudaEventCreateWithFlags(&ev_q, cudaEventDisableTiming));
		size_t total = 64;                   // the flag word, then the buffers (each 256-byte aligned)
		size_t offs[NBUF];
		for (int i = 0; i < NBUF; ++i) { offs[i] = total; total += (words_of(i) + 63) / 64 * 64; }
		CK(cudaMalloc(&dmem, total * 4));
		CK(cudaMemsetAsync(dmem, 0, total * 4, st));
		d_flag = dmem;
		for (int i = 0; i < NBUF; ++i) bufp[i] = dmem + offs[i];

		host.assign((size_t)AB_NW * n, 0);
		upload_twiddles();
		setup_device(pp);
	}
};

// ============================================================ batches
// A size class (K, pck, ln) of `cap` candidates with stacked buffers: buffer
// type i of slot s is at base[i] + s * (its words).  Each loaded slot is
// exposed as an ab_transform view (set1 / copy / mul / get work unchanged on
// it); the squarings of all slots run together (grid.z = slot) from a
// captured CUDA graph whose per-step, per-slot multipliers are uploaded
// before each launch.
struct ab_batch
{
	int device = 0;
	cudaStream_t st = nullptr;
	ab_params cls{};
	Geometry geo{};
	TConst tc{};
	RefConst rc{};
	size_t n = 0, w_ntt = 0, w_norm = 0;   // words of an NTT-form / normal-form buffer of one slot
	int cap = 0, max_steps = 0;
	u32 * mem = nullptr;
	u32 * d_flag = nullptr;
	u32 * base[ab_transform::NBUF] = {};
	CandConst * d_cand = nullptr;
	std::vector<CandConst> h_cand;
	u32 * d_ctrl = nullptr;            // per step: mult[cap] | act[cap] | snap[cap]
	u32 * h_ctrl[2] = {};              // page-locked staging, alternating between launches
	cudaEvent_t ctrl_done[2] = {};     // the upload out of h_ctrl[i] has completed
	int ctrl_i = 0;
	cudaEvent_t chunk_done = nullptr;  // the last chunk has completed
	std::vector<ab_transform *> views;
	cudaGraphExec_t gexec = nullptr;
	int g_steps = 0;
	uint64_t g_kernels = 0;
	int zl = 0;                        // slots the graph launches (grid.z): a power of two covering every live slot
	uint64_t launches = 0;

	~ab_batch()
	{
		for (ab_transform * v : views) delete v;
		if (gexec) cudaGraphExecDestroy(gexec);
		if (mem) cudaFree(mem);
		if (d_cand) cudaFree(d_cand);
		if (d_ctrl) cudaFree(d_ctrl);
		for (int i = 0; i < 2; ++i) { if (h_ctrl[i]) cudaFreeHost(h_ctrl[i]); if (ctrl_done[i]) cudaEventDestroy(ctrl_done[i]); }
		if (chunk_done) cudaEventDestroy(chunk_done);
		if (st) cudaStreamDestroy(st);
	}

	size_t slot_words(int i) const { return ab_transform::normal_buf(i) ? w_norm : w_ntt; }
	u32 * ctrl(int step, int part) const { return d_ctrl + ((size_t)step * 3 + part) * cap; }
	const uint2 * wf(bool q) const { return reinterpret_cast<const uint2 *>(base[q ? ab_transform::WQ : ab_transform::WR]); }
	const uint2 * wv(bool q) const { return q ? nullptr : reinterpret_cast<const uint2 *>(base[ab_transform::WRI]); }
	const uint2 * wc(bool q, bool inverse) const
	{
		return reinterpret_cast<const uint2 *>(base[ab_transform::WC]) + ((q ? 2 : 0) + (inverse ? 1 : 0)) * (cls.K + 1) * COLTW;
	}

	uint64_t recorded = 0;              // kernels recorded by rows()/cols() (graph nodes)
	int geo_version = 0;               // changes with the split (a mixed group then re-records)
	// when set, rows() and cols() append their passes here instead of launching
	struct Pass { bool row; RowJobs rj; ColJobs cj; int nj; };
	std::vector<Pass> * sink = nullptr;
	void rows(const RowJob & j0, const RowJob * j1 = nullptr)
	{
		RowJobs js; js.j[0] = j0; js.j[1] = j1 ? *j1 : j0;
		const int nj = j1 ? 2 : 1;
		if (sink) { Pass q{}; q.row = true; q.rj = js; q.nj = nj; sink->push_back(q); return; }
		if (geo.G > 0) { CK(launch_midpass(geo, tc, js, nj, st, zl, false)); ++recorded; }
		CK(launch_rowpass(geo, tc, js, nj, st, zl));
		++recorded;
		if (geo.G > 0 && j0.mode != ROW_FWD_ONLY) { CK(launch_midpass(geo, tc, js, nj, st, zl, true)); ++recorded; }
	}
	void cols(const ColJob & j0, const ColJob * j1 = nullptr)
	{
		ColJobs js; js.j[0] = j0; js.j[1] = j1 ? *j1 : j0;
		if (sink) { Pass q{}; q.row = false; q.cj = js; q.nj = j1 ? 2 : 1; sink->push_back(q); return; }
		CK(launch_colpass(geo, tc, js, j1 ? 2 : 1, st, zl));
		++recorded;
	}
	RowJob rj(u32 * x, int mode, bool q, const u32 * xp, const u32 * act) const
	{
		RowJob j; std::memset(&j, 0, sizeof(j));
		j.x = x; j.xp = xp; j.w = wf(q); j.wi = wv(q); j.mode = mode; j.stride = w_ntt; j.active = act;
		return j;
	}
	ColJob cj(const u32 * in, bool tr, bool q, const u32 * mult, const u32 * sub, int lower) const
	{
		ColJob j; std::memset(&j, 0, sizeof(j));
		j.in = in; j.transformed = tr ? 1 : 0;
		if (tr) { j.wi_in = wc(q, true); j.nega = q ? 1 : 0; }
		j.a = 1; j.mult = mult; j.sub = sub;
		j.lower = lower; j.stride_ntt = w_ntt; j.stride_norm = w_norm; j.cand = d_cand;
		return j;
	}
	void set_fwd(ColJob & j, u32 * q_out, u32 * r_out) const
	{
		j.out_fwd[0] = q_out; j.w_out[0] = q_out ? wc(true, false) : nullptr;
		j.out_fwd[1] = r_out; j.w_out[1] = r_out ? wc(false, false) : nullptr;
	}

	// squareMMGW (transformGPU.h:556-568) for every slot, `steps` times
	void record_steps(int steps)
	{
		using T = ab_transform;
		u32 * const aq0 = base[T::AQ0], * const ar0 = base[T::AR0], * const aq1 = base[T::AQ1], * const ar1 = base[T::AR1];
		{
			ColJob j = cj(base[T::REG0], false, false, ctrl(0, 1), nullptr, LOWER_NONE);
			set_fwd(j, aq0, ar0);
			cols(j);
		}
		for (int s = 0; s < steps; ++s)
		{
			const u32 * mult = ctrl(s, 0), * act = ctrl(s, 1), * snap = ctrl(s, 2);
			RowJob rq = rj(aq0, ROW_SQUARE, true, nullptr, act), rr = rj(ar0, ROW_SQUARE, false, nullptr, act);
			rows(rq, &rr);
			ColJob jq = cj(aq0, true, true, mult, nullptr, LOWER_NONE); jq.out_norm = base[T::TQ];
			ColJob jr = cj(ar0, true, false, mult, nullptr, LOWER_NONE); set_fwd(jr, nullptr, ar1);
			cols(jq, &jr);
			rows(rj(ar1, ROW_MUL, false, base[T::NIR], act));
			ColJob j1 = cj(ar1, true, false, act, nullptr, LOWER_R_ADD2); set_fwd(j1, aq1, nullptr);
			cols(j1);
			rows(rj(aq1, ROW_MUL, true, base[T::NQ], act));
			ColJob j2 = cj(aq1, true, true, act, base[T::TQ], LOWER_Q);
			j2.out_norm = base[T::REG0];
			set_fwd(j2, aq0, ar0);
			j2.out_snap = base[T::SNAP]; j2.snap_flag = snap;
			cols(j2);
		}
	}
};

// ============================================================ C ABI
namespace
{
template <typename F>
int guarded(F && f)
{
	try { f(); return AB_OK; }
	catch (const ab_error & e) { g_last_error = e.what(); return e.code; }
	catch (const std::exception & e) { g_last_error = e.what(); return AB_E_ARG; }
}

bool valid_reg(size_t r) { return r <= 2; }

void need_ready(const ab_transform * h)
{
	if (h == nullptr) throw ab_error(AB_E_ARG, "null handle");
	if (h->failed) throw ab_error(AB_E_INIT_FAILED, "gcd(N, R) != 1");
}
}

extern "C" {

int ab_probe(const uint64_t * Nl, size_t nlimbs, int32_t a, const ab_params * forced, ab_params * out, int * init_failed)
{
	return guarded([&] {
		if (Nl == nullptr || nlimbs == 0 || out == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
		mpz_t N, R, Ninv, f; mpz_inits(N, R, Ninv, f, nullptr);
		mpz_from_limbs(N, Nl, nlimbs);
		*out = forced ? *forced : select_params(N, a);
		if (init_failed) *init_failed = compute_R_Ninv(N, *out, R, Ninv, f) ? 0 : 1;
		mpz_clears(N, R, Ninv, f, nullptr);
	});
}

int ab_create(const uint64_t * Nl, size_t nlimbs, int32_t a, int device, const ab_params * forced, ab_transform ** out)
{
	if (out) *out = nullptr;
	ab_transform * h = nullptr;
	const int rc = guarded([&] {
		if (Nl == nullptr || nlimbs == 0 || out == nullptr || a < 1) throw ab_error(AB_E_ARG, "bad arguments");
		mpz_t N; mpz_init(N); mpz_from_limbs(N, Nl, nlimbs);
		h = new ab_transform();
		try { h->init(N, a, device, forced); }
		catch (...) { mpz_clear(N); throw; }
		mpz_clear(N);
	});
	if (rc != AB_OK) { delete h; return rc; }
	*out = h;
	return AB_OK;
}

void ab_destroy(ab_transform * h) { delete h; }

int ab_init_failed(const ab_transform * h) { return (h != nullptr && h->failed) ? 1 : 0; }

int ab_get_factor(const ab_transform * h, uint64_t * out, size_t cap, size_t * count)
{
	return guarded([&] {
		if (h == nullptr || count == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
		const mpz_srcptr z = h->failed ? h->factor : h->N;
		const size_t sz = mpz_size(z);
		if (sz > cap) throw ab_error(AB_E_CAPACITY, "output too small");
		for (size_t i = 0; i < sz; ++i) out[i] = mpz_getlimbn(z, (mp_size_t)i);
		*count = sz;
	});
}

int ab_info(const ab_transform * h, ab_params * out)
{
	return guarded([&] { if (h == nullptr || out == nullptr) throw ab_error(AB_E_ARG, "bad arguments"); *out = h->prm; });
}

int ab_set1(ab_transform * h)
{
	return guarded([&] { need_ready(h); h->copy(ab_transform::REG0, ab_transform::ONE); });
}

int ab_copy(ab_transform * h, size_t dst, size_t src)
{
	return guarded([&] {
		need_ready(h);
		if (!valid_reg(dst) || !valid_reg(src)) throw ab_error(AB_E_ARG, "register index");
		h->copy((int)dst, (int)src);
	});
}

int ab_square_mul(ab_transform * h, int32_t a)
{
	return guarded([&] {
		need_ready(h);
		if (a < 1) throw ab_error(AB_E_ARG, "multiplier a must be >= 1");
		h->square_mul((u32)a);
	});
}

int ab_square_mul_bits(ab_transform * h, const uint64_t * bits, size_t count, int32_t a)
{
	return guarded([&] {
		need_ready(h);
		if (a < 1 || (count != 0 && bits == nullptr)) throw ab_error(AB_E_ARG, "bad arguments");
		auto m_at = [&](size_t i) { return ((bits[i / 64] >> (i % 64)) & 1) ? (u32)a : 1u; };
		size_t i = 0;
		const size_t G = ab_transform::GRAPH_STEPS;
		if (!h->view && h->prof_used >= h->prof.size())
		{
			u32 m[ab_transform::GRAPH_STEPS];
			for (; i + G <= count; i += G)
			{
				for (size_t s = 0; s < G; ++s) m[s] = m_at(i + s);
				h->square_mul_graph(m);
			}
		}
		for (; i < count; ++i) h->square_mul(m_at(i));
	});
}

int ab_set_geometry(ab_transform * h, int row_levels)
{
	return guarded([&] {
		need_ready(h);
		if (h->view) throw ab_error(AB_E_ARG, "a batch slot takes the geometry of its batch");
		h->set_geometry(row_levels);
	});
}

int ab_set_overlap(ab_transform * h, int on)
{
	return guarded([&] {
		need_ready(h);
		if (h->view) throw ab_error(AB_E_ARG, "a batch slot runs on its batch's stream");
		CK(cudaStreamSynchronize(h->st));
		CK(cudaStreamSynchronize(h->st2));
		h->overlap = (on != 0);
		if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }   // captured with the old schedule
	});
}

int ab_get_geometry(const ab_transform * h, int * row_levels, int * col_levels)
{
	return guarded([&] {
		if (h == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
		if (row_levels) *row_levels = h->geo.LB;
		if (col_levels) *col_levels = h->geo.LA;
	});
}

int ab_mul(ab_transform * h, size_t dst, size_t src)
{
	return guarded([&] {
		need_ready(h);
		if (!valid_reg(dst) || !valid_reg(src)) throw ab_error(AB_E_ARG, "register index");
		h->mul((int)dst, (int)src);
	});
}

int ab_get(ab_transform * h, size_t src, uint64_t * out, size_t cap, size_t * count)
{
	return guarded([&] {
		need_ready(h);
		if (!valid_reg(src) || count == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
		mpz_t z; mpz_init(z);
		h->get((int)src, z);
		const size_t sz = mpz_size(z);
		if (sz > cap) { mpz_clear(z); throw ab_error(AB_E_CAPACITY, "output too small"); }
		for (size_t i = 0; i < sz; ++i) out[i] = mpz_getlimbn(z, (mp_size_t)i);
		*count = sz;
		mpz_clear(z);
	});
}

size_t ab_checkpoint_size(const ab_transform * h)
{
	return (h == nullptr) ? 0 : 8 + (size_t)8 * h->prm.K * h->n;
}

int ab_save_checkpoint(ab_transform * h, void * buf, size_t cap, size_t * written)
{
	return guarded([&] {
		need_ready(h);
		const size_t need = ab_checkpoint_size(h), K = (size_t)h->prm.K, n = h->n;
		if (buf == nullptr || cap < need) throw ab_error(AB_E_CAPACITY, "checkpoint buffer too small");
		u32 * o = static_cast<u32 *>(buf);
		o[0] = (u32)K; o[1] = (u32)n;
		// per prime k: plane k of Reg0 then plane k of Reg1 (transformGPU.h:626-641),
		// the reference's register words
		for (int r = 0; r < 2; ++r)
		{
			h->export_words(r == 0 ? ab_transform::REG0 : ab_transform::REG1);
			for (size_t k = 0; k < K; ++k)
				CK(cudaMemcpyAsync(o + 2 + 2 * k * n + r * n, h->b(ab_transform::XW) + k * n, n * 4, cudaMemcpyDeviceToHost, h->st));
		}
		CK(cudaStreamSynchronize(h->st));
		if (written) *written = need;
	});
}

int ab_read_checkpoint(ab_transform * h, const void * buf, size_t size)
{
	return guarded([&] {
		need_ready(h);
		const size_t K = (size_t)h->prm.K, n = h->n;
		if (buf == nullptr || size < 8) throw ab_error(AB_E_CHECKPOINT, "checkpoint too short");
		const u32 * in = static_cast<const u32 *>(buf);
		if (in[0] != K || in[1] != n || size < ab_checkpoint_size(h)) throw ab_error(AB_E_CHECKPOINT, "checkpoint does not match K or n");
		bool ok = true;
		for (int r = 0; r < 2; ++r)
		{
			for (size_t k = 0; k < K; ++k)
				CK(cudaMemcpyAsync(h->b(ab_transform::XW) + k * n, in + 2 + 2 * k * n + r * n, n * 4, cudaMemcpyHostToDevice, h->st));
			ok = h->import_words(r == 0 ? ab_transform::REG0 : ab_transform::REG1) && ok;
		}
		h->prefwd = false;
		if (!ok) throw ab_error(AB_E_CHECKPOINT, "checkpoint registers are not in normal form");
	});
}

void * ab_host_alloc(size_t bytes)
{
	void * p = nullptr;
	if (cudaMallocHost(&p, bytes) != cudaSuccess) { g_last_error = "cudaMallocHost failed"; return nullptr; }
	return p;
}

void ab_host_free(void * p) { if (p) cudaFreeHost(p); }

int ab_read_register(ab_transform * h, size_t reg, uint32_t * out, size_t cap_words)
{
	return guarded([&] {
		need_ready(h);
		if (!valid_reg(reg) || out == nullptr || cap_words < (size_t)h->prm.K * h->n) throw ab_error(AB_E_ARG, "bad arguments");
		h->export_words((int)reg);
		h->download(ab_transform::XW, out, (size_t)h->prm.K * h->n);
	});
}

int ab_write_register(ab_transform * h, size_t reg, const uint32_t * in, size_t nwords)
{
	return guarded([&] {
		need_ready(h);
		if (!valid_reg(reg) || in == nullptr || nwords != (size_t)h->prm.K * h->n) throw ab_error(AB_E_ARG, "bad arguments");
		h->upload(ab_transform::XW, in);
		if (!h->import_words((int)reg)) throw ab_error(AB_E_ARG, "the words are not a normal-form register");
	});
}

int ab_synchronize(ab_transform * h)
{
	return guarded([&] {
		if (h == nullptr) throw ab_error(AB_E_ARG, "null handle");
		if (h->st) CK(cudaStreamSynchronize(h->st));
	});
}

int ab_timer_start(ab_transform * h)
{
	return guarded([&] { need_ready(h); CK(cudaEventRecord(h->ev0, h->st)); });
}

int ab_timer_stop(ab_transform * h, float * ms)
{
	return guarded([&] {
		need_ready(h);
		CK(cudaEventRecord(h->ev1, h->st));
		CK(cudaEventSynchronize(h->ev1));
		CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
	});
}

const char * ab_last_error(void) { return g_last_error.c_str(); }

int ab_launch_count(const ab_transform * h, uint64_t * count)
{
	return guarded([&] { if (h == nullptr || count == nullptr) throw ab_error(AB_E_ARG, "bad arguments"); *count = h->launches; });
}

int ab_profile_square(ab_transform * h, int32_t a, float * ms, int cap, int * count)
{
	return guarded([&] {
		need_ready(h);
		if (ms == nullptr || count == nullptr || cap < 1) throw ab_error(AB_E_ARG, "bad arguments");
		if (h->prof.size() < (size_t)cap + 1)
		{
			for (cudaEvent_t e : h->prof) cudaEventDestroy(e);
			h->prof.assign((size_t)cap + 1, nullptr);
			for (auto & e : h->prof) CK(cudaEventCreate(&e));
		}
		h->prof_used = 0;                    // mark() records before every launch
		const bool ov = h->overlap;
		h->overlap = false;                  // one stream: launches in order
		h->split = true;                     // the same launches as the overlapped schedule
		try { h->square_mul((u32)a); }
		catch (...) { h->overlap = ov; h->split = false; throw; }
		h->overlap = ov;
		h->split = false;
		const size_t used = h->prof_used;
		h->prof_used = h->prof.size();       // recording off
		if (used == 0 || used > (size_t)cap) throw ab_error(AB_E_CAPACITY, "launch count exceeds cap");
		CK(cudaEventRecord(h->prof[used], h->st));
		CK(cudaEventSynchronize(h->prof[used]));
		for (size_t i = 0; i < used; ++i) CK(cudaEventElapsedTime(&ms[i], h->prof[i], h->prof[i + 1]));
		*count = (int)used;
	});
}

int ab_flush_l2(ab_transform * h, size_t bytes)
{
	return guarded([&] {
		need_ready(h);
		if (h->flush_buf == nullptr) CK(cudaMalloc(&h->flush_buf, bytes));
		CK(cudaMemsetAsync(h->flush_buf, (int)(h->launches & 0xff), bytes, h->st));
	});
}

int ab_square_mul_noalloc(ab_transform * h, uint32_t * reg, int32_t a)
{
	return guarded([&] {
		need_ready(h);
		if (reg == nullptr || a < 1) throw ab_error(AB_E_ARG, "null register or multiplier a < 1");
		const size_t n = h->n, ntt_words = (size_t)h->KP * n;
		if (ntt_words > AB_NOALLOC_MAX_WORDS || 2 * AB_NW * n > AB_NOALLOC_MAX_WORDS)
			throw ab_error(AB_E_CAPACITY, "ab_square_mul_noalloc: NTT length 2^" + std::to_string(h->prm.ln) +
				" exceeds the static scratch (at most 2^16 words per prime, " + std::to_string(AB_NOALLOC_MAX_WORDS) + " words per region)");
		u32 * const s = (h->noalloc != nullptr) ? h->noalloc : noalloc_scratch(h->device);
		u32 * const aq0 = s, * const ar0 = s + AB_NOALLOC_MAX_WORDS, * const aq1 = s + 2 * AB_NOALLOC_MAX_WORDS;
		u32 * const ar1 = s + 3 * AB_NOALLOC_MAX_WORDS, * const tq = s + 4 * AB_NOALLOC_MAX_WORDS;
		u32 * const x = tq + AB_NW * n, * const flag = s + 5 * AB_NOALLOC_MAX_WORDS;
		using T = ab_transform;
		// the caller's register words -> exact values in the scratch, then
		// squareMMGW (transformGPU.h:556-568) with every intermediate in the
		// static scratch, then back to the caller's register words.  Each
		// scratch word is written before it is read within the call, so
		// nothing needs clearing between calls.
		CK(launch_import(h->rc, reg, x, (u32)n, flag, h->st));
		ColJob j0 = h->cj_norm(x); h->set_fwd(j0, aq0, ar0); h->cols(j0);
		RowJob rq = h->rj(aq0, ROW_SQUARE, true), rr = h->rj(ar0, ROW_SQUARE, false);
		h->rows(rq, &rr);
		ColJob jq = h->cj_tr(aq0, true, (u32)a, nullptr, LOWER_NONE); jq.out_norm = tq;
		ColJob jr = h->cj_tr(ar0, false, (u32)a, nullptr, LOWER_NONE); h->set_fwd(jr, nullptr, ar1);
		h->cols(jq, &jr);
		h->rows(h->rj(ar1, ROW_MUL, false, h->b(T::NIR)));
		ColJob j1 = h->cj_tr(ar1, false, 1, nullptr, LOWER_R_ADD2); h->set_fwd(j1, aq1, nullptr); h->cols(j1);
		h->rows(h->rj(aq1, ROW_MUL, true, h->b(T::NQ)));
		ColJob j2 = h->cj_tr(aq1, true, 1, tq, LOWER_Q); j2.out_norm = x; h->cols(j2);
		CK(launch_export(h->rc, x, reg, (u32)n, h->st));
		h->launches += 2;
	});
}

int ab_inject_word(ab_transform * h, size_t reg, size_t index, int32_t delta)
{
	return guarded([&] {
		need_ready(h);
		if (!valid_reg(reg)) throw ab_error(AB_E_ARG, "register index");
		u32 * const w = h->b((int)reg) + index % (AB_NW * h->n);
		u32 v = 0;
		CK(cudaMemcpyAsync(&v, w, 4, cudaMemcpyDeviceToHost, h->st));
		CK(cudaStreamSynchronize(h->st));
		v += (u32)delta;
		CK(cudaMemcpyAsync(w, &v, 4, cudaMemcpyHostToDevice, h->st));
		CK(cudaStreamSynchronize(h->st));
		if (reg == 0) h->prefwd = false;
	});
}

int ab_diag_forward(ab_transform * h, int domain, const uint32_t * in, uint32_t * out)
{
	return guarded([&] {
		need_ready(h);
		using T = ab_transform;
		h->upload(T::XW, in);
		if (!h->import_words(T::TMP)) throw ab_error(AB_E_ARG, "input is not a normal-form register");
		if (domain) h->full_forward(h->b(T::TMP), h->b(T::AQ1), nullptr);
		else h->full_forward(h->b(T::TMP), nullptr, h->b(T::AQ1));
		h->download(T::AQ1, out, (size_t)h->KP * h->n);
		h->prefwd = false;
	});
}

int ab_diag_product(ab_transform * h, int domain, const uint32_t * in, const uint32_t * y, uint32_t a,
	const uint32_t * sub, int lower_mode, uint32_t * out)
{
	return guarded([&] {
		need_ready(h);
		using T = ab_transform;
		const bool q = domain != 0;
		auto load = [&](const uint32_t * words, int buf) {
			h->upload(T::XW, words);
			if (!h->import_words(buf)) throw ab_error(AB_E_ARG, "input is not a normal-form register");
		};
		load(in, T::TMP);
		if (y)
		{
			load(y, T::SNAP);
			h->full_forward(h->b(T::SNAP), q ? h->b(T::OPQ) : nullptr, q ? nullptr : h->b(T::OPR));
		}
		if (sub) load(sub, T::TQ);
		ColJob j = h->cj_norm(h->b(T::TMP));
		if (q) h->set_fwd(j, h->b(T::AQ1), nullptr); else h->set_fwd(j, nullptr, h->b(T::AQ1));
		h->cols(j);
		h->rows(h->rj(h->b(T::AQ1), y ? ROW_MUL : ROW_SQUARE, q, y ? h->b(q ? T::OPQ : T::OPR) : nullptr));
		ColJob c = h->cj_tr(h->b(T::AQ1), q, a, sub ? h->b(T::TQ) : nullptr, lower_mode);
		c.out_norm = h->b(T::TMP);
		h->cols(c);
		h->export_words(T::TMP);
		h->download(T::XW, out, (size_t)h->prm.K * h->n);
		h->prefwd = false;
	});
}


size_t ab_batch_slot_bytes(const ab_params * cls)
{
	if (cls == nullptr || cls->K < 2 || cls->K > 5) return 0;
	const size_t n = (size_t)1 << cls->ln, KP = (size_t)cls->K + 1;
	size_t w = 0;
	for (int i = 0; i < ab_transform::NSLOT; ++i) w += ab_transform::normal_buf(i) ? AB_NW * n : KP * n;
	return w * 4;
}

int ab_batch_create(int device, const ab_params * cls, int capacity, int max_steps, ab_batch ** out)
{
	if (out) *out = nullptr;
	ab_batch * b = nullptr;
	const int rc = guarded([&] {
		if (cls == nullptr || out == nullptr || capacity < 1 || max_steps < 1) throw ab_error(AB_E_ARG, "bad arguments");
		if (cls->K < 2 || cls->K > 5 || (size_t)cls->pck != get_s((size_t)cls->K)) throw ab_error(AB_E_ARG, "invalid size class");
		b = new ab_batch();
		b->device = device; b->cls = *cls; b->cap = capacity; b->max_steps = max_steps;
		if (!make_geometry(cls->ln, 0, b->geo)) throw ab_error(AB_E_UNSUPPORTED, "NTT length not supported");
		b->n = (size_t)1 << cls->ln;
		b->w_ntt = (size_t)(cls->K + 1) * b->n; b->w_norm = (size_t)AB_NW * b->n;
		CK(cudaSetDevice(device));
		// smaller classes at higher stream priority: their chunks are chains of
		// short, latency-bound launches, which otherwise queue behind the large
		// grids of the big classes sharing the GPU
		int least = 0, greatest = 0;
		CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
		const int prio = std::min(least, greatest + std::max(0, cls->ln - 12));
		CK(cudaStreamCreateWithPriority(&b->st, cudaStreamNonBlocking, prio));
		// the flag word, the per-slot buffers (slot-major within each type), then
		// the shared buffers: the reference words XW and the twiddle tables
		size_t total = 64, offs[ab_transform::NBUF];
		for (int i = 0; i < ab_transform::NBUF; ++i)
		{
			offs[i] = total;
			const size_t w = (i < ab_transform::NSLOT) ? b->slot_words(i) * capacity : ab_transform::words_of(i, cls->K, b->n);
			total += (w + 63) / 64 * 64;
		}
		CK(cudaMalloc(&b->mem, total * 4));
		CK(cudaMemsetAsync(b->mem, 0, total * 4, b->st));
		b->d_flag = b->mem;
		for (int i = 0; i < ab_transform::NBUF; ++i) b->base[i] = b->mem + offs[i];
		std::vector<uint2> wr, wri, wq, wcv;
		ab_transform::twiddle_tables(*cls, wr, wri, wq, wcv);
		CK(cudaMemcpyAsync(b->base[ab_transform::WR], wr.data(), wr.size() * sizeof(uint2), cudaMemcpyHostToDevice, b->st));
		CK(cudaMemcpyAsync(b->base[ab_transform::WRI], wri.data(), wri.size() * sizeof(uint2), cudaMemcpyHostToDevice, b->st));
		CK(cudaMemcpyAsync(b->base[ab_transform::WQ], wq.data(), wq.size() * sizeof(uint2), cudaMemcpyHostToDevice, b->st));
		CK(cudaMemcpyAsync(b->base[ab_transform::WC], wcv.data(), wcv.size() * sizeof(uint2), cudaMemcpyHostToDevice, b->st));
		CK(cudaMalloc(&b->d_cand, sizeof(CandConst) * capacity));
		b->h_cand.assign(capacity, CandConst{});
		for (auto & c : b->h_cand) c.lbase = 2;
		CK(cudaMemcpyAsync(b->d_cand, b->h_cand.data(), sizeof(CandConst) * capacity, cudaMemcpyHostToDevice, b->st));
		CK(cudaMalloc(&b->d_ctrl, (size_t)3 * max_steps * capacity * 4));
		CK(cudaMemsetAsync(b->d_ctrl, 0, (size_t)3 * max_steps * capacity * 4, b->st));
		for (int i = 0; i < 2; ++i)
		{
			CK(cudaMallocHost(&b->h_ctrl[i], (size_t)3 * max_steps * capacity * 4));
			CK(cudaEventCreateWithFlags(&b->ctrl_done[i], cudaEventDisableTiming));
			CK(cudaEventRecord(b->ctrl_done[i], b->st));
		}
		CK(cudaEventCreateWithFlags(&b->chunk_done, cudaEventDisableTiming));
		CK(cudaEventRecord(b->chunk_done, b->st));
		b->views.assign(capacity, nullptr);
		// constants of the class (the digit size comes from d_cand)
		ab_params p = *cls; p.lbase = 17;
		ab_transform::build_consts(p, b->geo, b->tc, b->rc);
		// kernel attributes before any capture
		RowJobs rjs{}; ColJobs cjs{};
		CK(launch_rowpass(b->geo, b->tc, rjs, 1, b->st, 0));
		CK(launch_colpass(b->geo, b->tc, cjs, 1, b->st, 0));
		CK(cudaStreamSynchronize(b->st));
	});
	if (rc != AB_OK) { delete b; return rc; }
	*out = b;
	return AB_OK;
}

void ab_batch_destroy(ab_batch * b) { delete b; }

namespace
{
// Host part of loading slots: parameters, R, N^-1 mod R (a gcd-sized GMP
// computation of a few hundred ms at millions of bits) and the register
// words, for several candidates at once on host threads.
void batch_prepare(int count, const uint64_t * const * Nl, const size_t * nlimbs, const int32_t * a,
                   std::vector<std::unique_ptr<ab_transform>> & views, std::vector<ab_transform::Prepared> & pp)
{
	views.clear();
	for (int i = 0; i < count; ++i) { views.emplace_back(new ab_transform()); views.back()->view = true; }
	pp.assign(count, ab_transform::Prepared());
	std::vector<std::string> err(count);
	std::vector<int> code(count, AB_OK);
	auto work = [&](int i) {
		try
		{
			mpz_t N; mpz_init(N); mpz_from_limbs(N, Nl[i], nlimbs[i]);
			try { views[i]->prepare(N, a[i], nullptr, pp[i]); }
			catch (...) { mpz_clear(N); throw; }
			mpz_clear(N);
		}
		catch (const ab_error & e) { code[i] = e.code; err[i] = e.what(); }
		catch (const std::exception & e) { code[i] = AB_E_ARG; err[i] = e.what(); }
	};
	const int nt = std::max(1, std::min(count, (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency()))));
	if (nt == 1) for (int i = 0; i < count; ++i) work(i);
	else
	{
		std::atomic<int> next{0};
		std::vector<std::thread> th;
		for (int t = 0; t < nt; ++t) th.emplace_back([&] { for (int i; (i = next.fetch_add(1)) < count;) work(i); });
		for (auto & x : th) x.join();
	}
	for (int i = 0; i < count; ++i) if (code[i] != AB_OK) throw ab_error(code[i], err[i]);
}

// A view's buffers: the slot's part of each per-slot buffer type, and the
// batch's shared buffers and stream.
void batch_attach(ab_batch * b, ab_transform * v, int slot)
{
	v->device = b->device; v->st = b->st; v->overlap = false;
	v->KP = b->cls.K + 1;
	v->d_flag = b->d_flag;
	for (int i = 0; i < ab_transform::NSLOT; ++i) v->bufp[i] = b->base[i] + (size_t)slot * b->slot_words(i);
	for (int i = ab_transform::NSLOT; i < ab_transform::NBUF; ++i) v->bufp[i] = b->base[i];
	v->host.assign(b->w_norm, 0);
}

// Device part: the slot's buffers, the transforms of N and N^-1, the constants
// of its digit size; the view then owns the slot.
void batch_install(ab_batch * b, int slot, std::unique_ptr<ab_transform> & vp, const ab_transform::Prepared & pp)
{
	ab_transform * v = vp.get();
	if (!v->failed && (v->prm.K != b->cls.K || v->prm.pck != b->cls.pck || v->prm.ln != b->cls.ln))
		throw ab_error(AB_E_ARG, "N does not belong to this size class");
	delete b->views[slot];
	b->views[slot] = nullptr;
	batch_attach(b, v, slot);
	v->noalloc = noalloc_scratch(b->device);
	v->use_geometry(b->geo);             // the batch's split, which the autotuner may have changed
	if (!v->failed)
	{
		v->setup_device(pp);
		CandConst & c = b->h_cand[slot];
		c.lbase = v->prm.lbase;
		CK(cudaMemcpyAsync(b->d_cand + slot, &c, sizeof(CandConst), cudaMemcpyHostToDevice, b->st));
		CK(cudaStreamSynchronize(b->st));
	}
	b->views[slot] = vp.release();
}
}

int ab_batch_load(ab_batch * b, int slot, const uint64_t * Nl, size_t nlimbs, int32_t a, int * init_failed)
{
	return ab_batch_load_many(b, 1, &slot, &Nl, &nlimbs, &a, init_failed);
}

int ab_batch_load_many(ab_batch * b, int count, const int * slots, const uint64_t * const * Nl, const size_t * nlimbs,
                       const int32_t * a, int * init_failed)
{
	return guarded([&] {
		if (b == nullptr || count < 0 || (count > 0 && (slots == nullptr || Nl == nullptr || nlimbs == nullptr || a == nullptr)))
			throw ab_error(AB_E_ARG, "bad arguments");
		for (int i = 0; i < count; ++i)
		{
			if (slots[i] < 0 || slots[i] >= b->cap || Nl[i] == nullptr || nlimbs[i] == 0 || a[i] < 1) throw ab_error(AB_E_ARG, "bad arguments");
			for (int j = 0; j < i; ++j) if (slots[j] == slots[i]) throw ab_error(AB_E_ARG, "a slot is named twice");
		}
		std::vector<std::unique_ptr<ab_transform>> views;
		std::vector<ab_transform::Prepared> pp;
		batch_prepare(count, Nl, nlimbs, a, views, pp);
		for (int i = 0; i < count; ++i)
		{
			if (init_failed) init_failed[i] = views[i]->failed ? 1 : 0;
			batch_install(b, slots[i], views[i], pp[i]);
		}
	});
}

struct ab_prepared
{
	std::unique_ptr<ab_transform> v;
	ab_transform::Prepared pp;
};

int ab_batch_prepare(const uint64_t * Nl, size_t nlimbs, int32_t a, ab_prepared ** out, ab_params * params, int * init_failed)
{
	if (out) *out = nullptr;
	ab_prepared * p = nullptr;
	const int rc = guarded([&] {
		if (Nl == nullptr || nlimbs == 0 || a < 1 || out == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
		std::vector<std::unique_ptr<ab_transform>> views;
		std::vector<ab_transform::Prepared> pp;
		batch_prepare(1, &Nl, &nlimbs, &a, views, pp);
		p = new ab_prepared();
		p->v = std::move(views[0]);
		p->pp = std::move(pp[0]);
		if (params) *params = p->v->prm;
		if (init_failed) *init_failed = p->v->failed ? 1 : 0;
	});
	if (rc != AB_OK) { delete p; return rc; }
	*out = p;
	return AB_OK;
}

int ab_prepared_factor(const ab_prepared * p, uint64_t * out, size_t cap, size_t * count)
{
	return guarded([&] {
		if (p == nullptr || count == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
		if (!p->v->failed) throw ab_error(AB_E_ARG, "gcd(N, R) = 1: no factor");
		const mpz_srcptr z = p->v->factor;
		const size_t sz = mpz_size(z);
		if (sz > cap) throw ab_error(AB_E_CAPACITY, "output too small");
		for (size_t i = 0; i < sz; ++i) out[i] = mpz_getlimbn(z, (mp_size_t)i);
		*count = sz;
	});
}

size_t ab_prepared_bytes(const ab_prepared * p)
{
	if (p == nullptr) return 0;
	return (p->pp.wN.size() + p->pp.wNinv.size() + p->pp.wOne.size()) * sizeof(u32);
}

void ab_prepared_destroy(ab_prepared * p) { delete p; }

int ab_batch_install(ab_batch * b, int slot, ab_prepared * p)
{
	std::unique_ptr<ab_prepared> own(p);
	return guarded([&] {
		if (b == nullptr || p == nullptr || slot < 0 || slot >= b->cap) throw ab_error(AB_E_ARG, "bad arguments");
		batch_install(b, slot, own->v, own->pp);
	});
}

int ab_batch_ready(const ab_batch * b)
{
	if (b == nullptr) return AB_E_ARG;
	for (int i = 0; i < 2; ++i)
	{
		const cudaError_t e = cudaEventQuery(i == 0 ? b->chunk_done : b->ctrl_done[b->ctrl_i]);
		if (e == cudaSuccess) return 2 - i;
		if (e != cudaErrorNotReady)
		{
			g_last_error = std::string("ab_batch_ready: ") + cudaGetErrorString(e);
			return AB_E_CUDA;
		}
	}
	return 0;
}

ab_transform * ab_batch_slot(ab_batch * b, int slot)
{
	if (b == nullptr || slot < 0 || slot >= b->cap) return nullptr;
	return b->views[slot];
}

int ab_batch_clone(ab_batch * b, int dst, int src)
{
	return guarded([&] {
		if (b == nullptr || dst < 0 || dst >= b->cap || src < 0 || src >= b->cap || dst == src || b->views[src] == nullptr)
			throw ab_error(AB_E_ARG, "bad arguments");
		const ab_transform * s = b->views[src];
		delete b->views[dst];
		b->views[dst] = nullptr;
		ab_transform * v = new ab_transform();
		v->view = true;
		mpz_set(v->N, s->N); mpz_set(v->factor, s->factor);
		v->prm = s->prm; v->n = s->n; v->geo = s->geo; v->tc = s->tc; v->rc = s->rc; v->failed = s->failed;
		batch_attach(b, v, dst);
		v->noalloc = s->noalloc;
		for (int i = 0; i < ab_transform::NSLOT; ++i)
			CK(cudaMemcpyAsync(v->bufp[i], s->bufp[i], b->slot_words(i) * 4, cudaMemcpyDeviceToDevice, b->st));
		b->h_cand[dst] = b->h_cand[src];
		CK(cudaMemcpyAsync(b->d_cand + dst, &b->h_cand[dst], sizeof(CandConst), cudaMemcpyHostToDevice, b->st));
		CK(cudaStreamSynchronize(b->st));
		b->views[dst] = v;
	});
}

int ab_batch_release(ab_batch * b, int slot)
{
	return guarded([&] {
		if (b == nullptr || slot < 0 || slot >= b->cap) throw ab_error(AB_E_ARG, "bad arguments");
		delete b->views[slot];
		b->views[slot] = nullptr;
	});
}

int ab_batch_gl_mul(ab_batch * b, int slot)
{
	return guarded([&] {
		if (b == nullptr || slot < 0 || slot >= b->cap || b->views[slot] == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
		need_ready(b->views[slot]);
		b->views[slot]->mul(ab_transform::REG1, ab_transform::SNAP);
	});
}

int ab_batch_steps(ab_batch * b, int steps, const uint32_t * mult, const uint8_t * snap)
{
	return guarded([&] {
		if (b == nullptr || mult == nullptr || steps < 1 || steps > b->max_steps) throw ab_error(AB_E_ARG, "bad arguments");
		const int cap = b->cap;
		// launch only as many slots as the highest one that steps: idle slots above
		// it cost a launch of empty blocks per pass
		int top = 0;
		for (int c = 0; c < cap; ++c)
			if (b->views[c] != nullptr && !b->views[c]->failed)
				for (int s = 0; s < steps; ++s) if (mult[(size_t)s * cap + c] != 0u) { top = c + 1; break; }
		int zl = 1;
		while (zl < top) zl <<= 1;
		zl = std::min(zl, cap);
		// the staging buffer used two launches ago must have been uploaded
		const int hi = b->ctrl_i;
		CK(cudaEventSynchronize(b->ctrl_done[hi]));
		u32 * const hc = b->h_ctrl[hi];
		for (int s = 0; s < steps; ++s)
			for (int c = 0; c < cap; ++c)
			{
				const bool live = b->views[c] != nullptr && !b->views[c]->failed;
				const u32 m = live ? mult[(size_t)s * cap + c] : 0u;
				hc[((size_t)s * 3 + 0) * cap + c] = m;
				hc[((size_t)s * 3 + 1) * cap + c] = (m != 0u) ? 1u : 0u;
				hc[((size_t)s * 3 + 2) * cap + c] = (snap != nullptr && m != 0u && snap[(size_t)s * cap + c]) ? 1u : 0u;
			}
		CK(cudaMemcpyAsync(b->d_ctrl, hc, (size_t)3 * steps * cap * 4, cudaMemcpyHostToDevice, b->st));
		CK(cudaEventRecord(b->ctrl_done[hi], b->st));
		b->ctrl_i ^= 1;
		if (b->gexec == nullptr || b->g_steps != steps || b->zl != zl)
		{
			if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
			b->zl = zl;
			cudaGraph_t g = nullptr;
			b->recorded = 0;
			CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
			try { b->record_steps(steps); }
			catch (...) { cudaStreamEndCapture(b->st, &g); if (g) cudaGraphDestroy(g); throw; }
			CK(cudaStreamEndCapture(b->st, &g));
			const cudaError_t e = cudaGraphInstantiate(&b->gexec, g, 0);
			cudaGraphDestroy(g);
			CK(e);
			b->g_steps = steps;
			b->g_kernels = b->recorded;
		}
		CK(cudaGraphLaunch(b->gexec, b->st));
		CK(cudaEventRecord(b->chunk_done, b->st));
		b->launches += b->g_kernels;                  // kernels of the graph
		for (ab_transform * v : b->views) if (v) v->prefwd = false;
	});
}

int ab_batch_set_geometry(ab_batch * b, int lb)
{
	return guarded([&] {
		if (b == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
		Geometry g;
		if (!make_geometry(b->cls.ln, lb, g)) throw ab_error(AB_E_ARG, "geometry not available for this length");
		CK(cudaStreamSynchronize(b->st));
		b->geo = g;
		++b->geo_version;
		apply_geometry(b->tc, g);
		for (ab_transform * v : b->views) if (v) { v->use_geometry(g); v->prefwd = false; }
		RowJobs rjs{}; ColJobs cjs{};
		CK(launch_rowpass(b->geo, b->tc, rjs, 1, b->st, 0));
		CK(launch_colpass(b->geo, b->tc, cjs, 1, b->st, 0));
		if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
	});
}

// Splits chosen by ab_batch_autotune in this process, by (K, ln, capacity).
namespace
{
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tuned;

void ok_or_throw(int rc) { if (rc != AB_OK) throw ab_error(rc, ab_last_error()); }
}

int ab_batch_autotune(ab_batch * b, int src, int steps, int * row_levels)
{
	return guarded([&] {
		if (b == nullptr || src < 0 || src >= b->cap || b->views[src] == nullptr || b->views[src]->failed || steps < 1 || steps > b->max_steps)
			throw ab_error(AB_E_ARG, "bad arguments");
		const auto key = std::make_tuple(b->cls.K, b->cls.ln, b->cap);
		int best = 0;
		{
			std::lock_guard<std::mutex> lock(g_tune_mu);
			auto it = g_tuned.find(key);
			if (it != g_tuned.end()) best = it->second;
		}
		if (best == 0)
		{
			// copies of `src` fill the empty slots; only they step (src and the
			// other loaded slots keep their registers)
			std::vector<int> tmp;
			for (int c = 0; c < b->cap; ++c) if (b->views[c] == nullptr) { ok_or_throw(ab_batch_clone(b, c, src)); tmp.push_back(c); }
			std::vector<u32> mult((size_t)steps * b->cap, 0u);
			for (int s = 0; s < steps; ++s) for (int c : tmp) mult[(size_t)s * b->cap + c] = 1u;
			cudaEvent_t e0 = nullptr, e1 = nullptr;
			float best_ms = 0;
			try
			{
				CK(cudaEventCreate(&e0)); CK(cudaEventCreate(&e1));
				const int L = b->cls.ln - 1;
				for (int lb = 4; lb <= 13 && !tmp.empty(); ++lb)
				{
					Geometry g;
					if (!make_geometry(b->cls.ln, lb, g) || L - lb > 6) continue;
					ok_or_throw(ab_batch_set_geometry(b, lb));
					ok_or_throw(ab_batch_steps(b, steps, mult.data(), nullptr));     // capture and warm-up
					CK(cudaEventRecord(e0, b->st));
					for (int r = 0; r < 2; ++r) ok_or_throw(ab_batch_steps(b, steps, mult.data(), nullptr));
					CK(cudaEventRecord(e1, b->st));
					CK(cudaEventSynchronize(e1));
					float ms = 0; CK(cudaEventElapsedTime(&ms, e0, e1));
					if (best == 0 || ms < best_ms) { best = lb; best_ms = ms; }
				}
			}
			catch (...)
			{
				for (int c : tmp) ab_batch_release(b, c);
				if (e0) cudaEventDestroy(e0);
				if (e1) cudaEventDestroy(e1);
				throw;
			}
			for (int c : tmp) ok_or_throw(ab_batch_release(b, c));
			cudaEventDestroy(e0); cudaEventDestroy(e1);
			if (best == 0) best = b->geo.LB;      // batch full: keep the current split
			else
			{
				std::lock_guard<std::mutex> lock(g_tune_mu);
				g_tuned[key] = best;
			}
		}
		if (best != b->geo.LB) ok_or_throw(ab_batch_set_geometry(b, best));
		if (row_levels) *row_levels = best;
	});
}

int ab_batch_synchronize(ab_batch * b)
{
	return guarded([&] { if (b == nullptr) throw ab_error(AB_E_ARG, "bad arguments"); CK(cudaStreamSynchronize(b->st)); });
}

int ab_batch_launch_count(const ab_batch * b, uint64_t * count)
{
	return guarded([&] { if (b == nullptr || count == nullptr) throw ab_error(AB_E_ARG, "bad arguments"); *count = b->launches; });
}

}

// ============================================================ mixed-size groups
// Batches of different size classes squared together: each pass of a chunk
// (the initial forward column levels, then per squaring the six row and
// column passes of the batch schedule) is one launch over the candidates of
// every class, driven by a device table of per-class jobs (FusedRowPass /
// FusedColPass).  The passes are the ones each batch would launch itself,
// recorded through its sink, so a slot's results do not depend on the group.
struct ab_mixed
{
	int device = 0;
	cudaStream_t st = nullptr;
	std::vector<ab_batch *> b;
	int max_steps = 0;
	TConst * d_tc = nullptr;
	FusedRowPass * d_row = nullptr;
	FusedColPass * d_col = nullptr;
	std::vector<u32 *> h_ctrl[2];      // per batch: page-locked control staging, alternating
	cudaEvent_t ctrl_done[2] = {};
	int ctrl_i = 0;
	cudaEvent_t chunk_done = nullptr, ev_join = nullptr;
	cudaGraphExec_t gexec = nullptr;
	int g_steps = 0;
	std::vector<int> g_zl, g_ver;
	uint64_t g_kernels = 0, launches = 0;

	~ab_mixed()
	{
		if (gexec) cudaGraphExecDestroy(gexec);
		if (d_tc) cudaFree(d_tc);
		if (d_row) cudaFree(d_row);
		if (d_col) cudaFree(d_col);
		for (int i = 0; i < 2; ++i)
		{
			for (u32 * h : h_ctrl[i]) if (h) cudaFreeHost(h);
			if (ctrl_done[i]) cudaEventDestroy(ctrl_done[i]);
		}
		if (chunk_done) cudaEventDestroy(chunk_done);
		if (ev_join) cudaEventDestroy(ev_join);
		if (st) cudaStreamDestroy(st);
	}

	// records the passes of `steps` squarings of every batch and captures them
	// as fused launches
	void capture(int steps, const std::vector<int> & zl)
	{
		const int nc = (int)b.size();
		std::vector<std::vector<ab_batch::Pass>> lists(nc);
		for (int i = 0; i < nc; ++i)
		{
			b[i]->sink = &lists[i];
			try { b[i]->record_steps(steps); }
			catch (...) { b[i]->sink = nullptr; throw; }
			b[i]->sink = nullptr;
		}
		const size_t np = lists[0].size();
		for (int i = 1; i < nc; ++i)
		{
			if (lists[i].size() != np) throw ab_error(AB_E_ARG, "batches of a group record different schedules");
			for (size_t q = 0; q < np; ++q)
				if (lists[i][q].row != lists[0][q].row) throw ab_error(AB_E_ARG, "batches of a group record different schedules");
		}
		std::vector<FusedRowPass> hr;
		std::vector<FusedColPass> hc;
		std::vector<u32> ctas;
		size_t smem_row = 0, smem_col = 0;
		for (int i = 0; i < nc; ++i)
		{
			smem_row = std::max(smem_row, fused_rowpass_smem(b[i]->geo.LB + 1));
			smem_col = std::max(smem_col, colpass_smem(b[i]->geo, b[i]->cls.K + 1));
		}
		for (size_t q = 0; q < np; ++q)
		{
			if (lists[0][q].row)
			{
				FusedRowPass f; std::memset(&f, 0, sizeof(f));
				f.nclass = nc;
				for (int i = 0; i < nc; ++i)
				{
					const ab_batch & x = *b[i];
					f.nbx[i] = (u32)(x.cls.K + 1) * x.geo.HR;
					f.njobs[i] = (u32)lists[i][q].nj;
					f.log_r[i] = x.geo.LB + 1;
					f.jobs[i] = lists[i][q].rj;
					f.begin[i + 1] = f.begin[i] + f.nbx[i] * f.njobs[i] * (u32)zl[i];
				}
				ctas.push_back(f.begin[nc]);
				hr.push_back(f);
			}
			else
			{
				FusedColPass f; std::memset(&f, 0, sizeof(f));
				f.nclass = nc;
				for (int i = 0; i < nc; ++i)
				{
					const ab_batch & x = *b[i];
					f.nbx[i] = x.geo.RC / (u32)x.geo.C;
					f.njobs[i] = (u32)lists[i][q].nj;
					f.sel[i] = x.geo.LA * 8 + x.cls.K;
					f.jobs[i] = lists[i][q].cj;
					f.begin[i + 1] = f.begin[i] + f.nbx[i] * f.njobs[i] * (u32)zl[i];
				}
				ctas.push_back(f.begin[nc]);
				hc.push_back(f);
			}
		}
		if (hr.size() > (size_t)3 * max_steps || hc.size() > (size_t)3 * max_steps + 1) throw ab_error(AB_E_ARG, "schedule longer than the group's tables");
		std::vector<TConst> tcs(nc);
		for (int i = 0; i < nc; ++i) tcs[i] = b[i]->tc;
		CK(cudaMemcpyAsync(d_tc, tcs.data(), sizeof(TConst) * nc, cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(d_row, hr.data(), sizeof(FusedRowPass) * hr.size(), cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(d_col, hc.data(), sizeof(FusedColPass) * hc.size(), cudaMemcpyHostToDevice, st));
		CK(cudaStreamSynchronize(st));
		// kernel attributes before the capture
		CK(launch_fused_rowpass(d_row, d_tc, 0, smem_row, st));
		CK(launch_fused_colpass(d_col, d_tc, 0, smem_col, st));
		if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
		cudaGraph_t g = nullptr;
		g_kernels = 0;
		CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		try
		{
			size_t ri = 0, ci = 0;
			for (size_t q = 0; q < np; ++q)
			{
				if (ctas[q] == 0) { (lists[0][q].row ? ri : ci)++; continue; }
				if (lists[0][q].row) CK(launch_fused_rowpass(d_row + ri++, d_tc, ctas[q], smem_row, st));
				else CK(launch_fused_colpass(d_col + ci++, d_tc, ctas[q], smem_col, st));
				++g_kernels;
			}
		}
		catch (...) { cudaStreamEndCapture(st, &g); if (g) cudaGraphDestroy(g); throw; }
		CK(cudaStreamEndCapture(st, &g));
		const cudaError_t e = cudaGraphInstantiate(&gexec, g, 0);
		cudaGraphDestroy(g);
		CK(e);
		g_steps = steps;
		g_zl = zl;
		g_ver.clear();
		for (ab_batch * x : b) g_ver.push_back(x->geo_version);
	}
};

extern "C" {

int ab_mixed_create(ab_batch * const * batches, int count, int max_steps, ab_mixed ** out)
{
	if (out) *out = nullptr;
	ab_mixed * m = nullptr;
	const int rc = guarded([&] {
		if (batches == nullptr || out == nullptr || count < 1 || count > AB_FUSE_MAXC || max_steps < 1) throw ab_error(AB_E_ARG, "bad arguments");
		for (int i = 0; i < count; ++i)
		{
			const ab_batch * x = batches[i];
			if (x == nullptr || x->device != batches[0]->device || max_steps > x->max_steps) throw ab_error(AB_E_ARG, "bad arguments");
			if (x->geo.G > 0) throw ab_error(AB_E_UNSUPPORTED, "a group takes lengths up to 2^20");
			for (int j = 0; j < i; ++j) if (batches[j] == x) throw ab_error(AB_E_ARG, "a batch is named twice");
		}
		m = new ab_mixed();
		m->device = batches[0]->device;
		m->b.assign(batches, batches + count);
		m->max_steps = max_steps;
		CK(cudaSetDevice(m->device));
		int least = 0, greatest = 0;
		CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
		CK(cudaStreamCreateWithPriority(&m->st, cudaStreamNonBlocking, greatest));
		CK(cudaMalloc(&m->d_tc, sizeof(TConst) * count));
		CK(cudaMalloc(&m->d_row, sizeof(FusedRowPass) * 3 * max_steps));
		CK(cudaMalloc(&m->d_col, sizeof(FusedColPass) * (3 * max_steps + 1)));
		for (int i = 0; i < 2; ++i)
		{
			for (ab_batch * x : m->b)
			{
				u32 * h = nullptr;
				CK(cudaMallocHost(&h, (size_t)3 * max_steps * x->cap * 4));
				m->h_ctrl[i].push_back(h);
			}
			CK(cudaEventCreateWithFlags(&m->ctrl_done[i], cudaEventDisableTiming));
			CK(cudaEventRecord(m->ctrl_done[i], m->st));
		}
		CK(cudaEventCreateWithFlags(&m->chunk_done, cudaEventDisableTiming));
		CK(cudaEventCreateWithFlags(&m->ev_join, cudaEventDisableTiming));
		CK(cudaEventRecord(m->chunk_done, m->st));
	});
	if (rc != AB_OK) { delete m; return rc; }
	*out = m;
	return AB_OK;
}

void ab_mixed_destroy(ab_mixed * m)
{
	if (m) cudaStreamSynchronize(m->st);
	delete m;
}

int ab_mixed_steps(ab_mixed * m, int steps, const uint32_t * const * mult, const uint8_t * const * snap)
{
	return guarded([&] {
		if (m == nullptr || mult == nullptr || steps < 1 || steps > m->max_steps) throw ab_error(AB_E_ARG, "bad arguments");
		const int nc = (int)m->b.size();
		std::vector<int> zl(nc, 0);
		bool any = false;
		for (int i = 0; i < nc; ++i)
		{
			const ab_batch & x = *m->b[i];
			if (mult[i] == nullptr) throw ab_error(AB_E_ARG, "bad arguments");
			int top = 0;
			for (int c = 0; c < x.cap; ++c)
				if (x.views[c] != nullptr && !x.views[c]->failed)
					for (int s = 0; s < steps; ++s) if (mult[i][(size_t)s * x.cap + c] != 0u) { top = c + 1; break; }
			int z = (top > 0) ? 1 : 0;
			while (z < top) z <<= 1;
			zl[i] = std::min(z, x.cap);
			any |= top > 0;
		}
		if (!any) return;
		// control words: the staging used two chunks ago must have been uploaded
		const int hi = m->ctrl_i;
		CK(cudaEventSynchronize(m->ctrl_done[hi]));
		for (int i = 0; i < nc; ++i)
		{
			ab_batch & x = *m->b[i];
			u32 * const hc = m->h_ctrl[hi][i];
			const int cap = x.cap;
			for (int s = 0; s < steps; ++s)
				for (int c = 0; c < cap; ++c)
				{
					const bool live = x.views[c] != nullptr && !x.views[c]->failed;
					const u32 mv = live ? mult[i][(size_t)s * cap + c] : 0u;
					hc[((size_t)s * 3 + 0) * cap + c] = mv;
					hc[((size_t)s * 3 + 1) * cap + c] = (mv != 0u) ? 1u : 0u;
					hc[((size_t)s * 3 + 2) * cap + c] = (snap != nullptr && snap[i] != nullptr && mv != 0u && snap[i][(size_t)s * cap + c]) ? 1u : 0u;
				}
			// the batch's own work (loads, Gerbicz-Li products, reads) comes first
			CK(cudaEventRecord(m->ev_join, x.st));
			CK(cudaStreamWaitEvent(m->st, m->ev_join, 0));
			CK(cudaMemcpyAsync(x.d_ctrl, hc, (size_t)3 * steps * cap * 4, cudaMemcpyHostToDevice, m->st));
		}
		CK(cudaEventRecord(m->ctrl_done[hi], m->st));
		m->ctrl_i ^= 1;
		bool same = (m->gexec != nullptr && m->g_steps == steps && m->g_zl == zl);
		for (int i = 0; same && i < nc; ++i) same = (m->g_ver[i] == m->b[i]->geo_version);
		if (!same) m->capture(steps, zl);
		CK(cudaGraphLaunch(m->gexec, m->st));
		CK(cudaEventRecord(m->chunk_done, m->st));
		m->launches += m->g_kernels;
		for (ab_batch * x : m->b)
		{
			CK(cudaStreamWaitEvent(x->st, m->chunk_done, 0));
			for (ab_transform * v : x->views) if (v) v->prefwd = false;
		}
	});
}

int ab_mixed_ready(const ab_mixed * m)
{
	if (m == nullptr) return AB_E_ARG;
	for (int i = 0; i < 2; ++i)
	{
		const cudaError_t e = cudaEventQuery(i == 0 ? m->chunk_done : m->ctrl_done[m->ctrl_i]);
		if (e == cudaSuccess) return 2 - i;
		if (e != cudaErrorNotReady)
		{
			g_last_error = std::string("ab_mixed_ready: ") + cudaGetErrorString(e);
			return AB_E_CUDA;
		}
	}
	return 0;
}

int ab_mixed_synchronize(ab_mixed * m)
{
	return guarded([&] { if (m == nullptr) throw ab_error(AB_E_ARG, "bad arguments"); CK(cudaStreamSynchronize(m->st)); });
}

int ab_mixed_launch_count(const ab_mixed * m, uint64_t * count)
{
	return guarded([&] { if (m == nullptr || count == nullptr) throw ab_error(AB_E_ARG, "bad arguments"); *count = m->launches; });
}

}
