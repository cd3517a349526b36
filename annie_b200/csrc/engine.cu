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
// (src/transformGPU.h:79-89).
const u32 PRIMES[14] = {
	(125u << 25) + 1, (243u << 24) + 1, (235u << 24) + 1, (29u << 27) + 1,
	(13u << 28) + 1, (193u << 24) + 1, (3u << 30) + 1, (43u << 26) + 1,
	(171u << 24) + 1, (81u << 25) + 1, (157u << 24) + 1, (151u << 24) + 1,
	(37u << 26) + 1, (17u << 27) + 1 };
const u32 PRIMROOTS[14] = { 3, 7, 3, 3, 3, 3, 5, 3, 35, 5, 3, 3, 3, 3 };

struct HostZp
{
	u32 p, q, one, rsq;
	explicit HostZp(u32 pp) : p(pp)
	{
		q = 1; for (int i = 0; i < 6; ++i) q *= 2 - p * q;      // p^-1 mod 2^32 (Newton)
		one = (u32)(((u64)1 << 32) % p);
		rsq = (u32)(((u64)one * one) % p);
	}
	u32 add(u32 a, u32 b) const { return a + b - ((a >= p - b) ? p : 0); }
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

size_t bitrev(size_t i, size_t n)
{
	size_t r = 0;
	for (size_t k = n, j = i; k > 1; k /= 2, j /= 2) r = (2 * r) | (j % 2);
	return r;
}

// Twiddles w[S + bitrev(j, S)], S = n/4 .. 1, inverse at +n/2; w[0] is the
// Montgomery form of w[1].  Domain R (x^n - 1) uses roots of unity of order
// 2S, domain Q (x^n + 1) the twisted roots of order 4S (transformGPU.h:117-160).
void make_roots(u32 * w, int ln, int k, bool domain_q)
{
	const HostZp z(PRIMES[k]);
	const size_t n = (size_t)1 << ln;
	u32 * wi = w + n / 2;
	auto primroot_n = [&](int l) { return z.pow(z.to_mont(PRIMROOTS[k]), (z.p - 1) >> l); };
	if (!domain_q)
	{
		u32 sr = primroot_n(ln - 1), sri = z.inv(sr);
		for (size_t s = n / 4; s >= 1; s /= 2)
		{
			u32 t = z.one, ti = z.one;
			for (size_t j = 0; j < s; ++j) { const size_t jr = bitrev(j, s); w[s + jr] = t; wi[s + jr] = ti; t = z.mul(t, sr); ti = z.mul(ti, sri); }
			sr = z.mul(sr, sr); sri = z.mul(sri, sri);
		}
	}
	else
	{
		u32 sr2 = primroot_n(ln), sr2i = z.inv(sr2);
		for (size_t s = n / 4; s >= 1; s /= 2)
		{
			const u32 sr = z.mul(sr2, sr2), sri = z.mul(sr2i, sr2i);
			u32 t = sr2, ti = sr2i;
			for (size_t j = 0; j < s; ++j) { const size_t jr = bitrev(j, s); w[s + jr] = t; wi[s + jr] = ti; t = z.mul(t, sr); ti = z.mul(ti, sri); }
			sr2 = sr; sr2i = sri;
		}
	}
	w[0] = z.to_mont(w[1]);
	wi[0] = 0;
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
// Work buffers of ab_square_mul_noalloc: five registers of at most
// AB_NOALLOC_MAX_WORDS words each (10 MiB), in a static device array that
// every GPU loading this library holds until the process exits.  Host code
// cannot use the symbol as an address: the device address is fetched with
// cudaGetSymbolAddress, with that device current, once per device -- when a
// transform or a batch is created there, so that the entry point itself only
// queues kernels.
#define AB_NOALLOC_MAX_WORDS (1u << 19)
#define AB_NOALLOC_MAX_DEVICES 64
static __device__ __align__(256) u32 g_noalloc_scratch[5 * AB_NOALLOC_MAX_WORDS];

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
	enum Buf { REG0 = 0, REG1, REG2, ONE, TQ, NQ, NIR, OPQ, OPR, AQ0, AQ1, AR0, AR1, TMP, SNAP, WR, WQ, NBUF };

	int device = 0;
	cudaStream_t st = nullptr;
	cudaStream_t st2 = nullptr;          // Q-domain chain, joined before the carry-sub
	cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_fork = nullptr, ev_q = nullptr;
	bool overlap = true;                 // run the Q chain on st2 (off for per-launch profiling)
	bool split = false;                  // without overlap: still one launch per domain
	ab_params prm{};
	size_t n = 0;
	Geometry geo{};
	TConst tc{};
	bool failed = false;
	mpz_t N, factor;
	u32 * dmem = nullptr;
	bool prefwd = false;     // AQ0/AR0 hold the first forward levels of REG0
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

	void build_consts()
	{
		const int K = prm.K;
		std::memset(&tc, 0, sizeof(tc));
		tc.K = K; tc.pck = prm.pck; tc.lbase = prm.lbase; tc.ln = prm.ln;
		tc.n = (u32)n; tc.R = geo.R; tc.H = geo.H; tc.LA = geo.LA; tc.LB = geo.LB;
		for (int k = 0; k < K; ++k)
		{
			const HostZp z(PRIMES[k]);
			tc.p[k] = z.p; tc.q[k] = z.q; tc.rsq[k] = z.rsq;
			tc.norm[k] = z.p - ((z.p - 1) >> (prm.ln - 1));
			const u32 base = (u32)((1ull << prm.lbase) % z.p);
			tc.rbase[k] = z.to_mont(base);
			u32 bp = 1; for (int l = 0; l < prm.pck; ++l) bp = (u32)(((u64)bp * base) % z.p);
			tc.rbase_pck[k] = bp;
			const u32 b2 = (u32)(((u64)base * base) % z.p);
			tc.b2m[k] = z.to_mont(b2); tc.b2mq[k] = tc.b2m[k] * z.q;
			for (int j = k + 1; j < K; ++j)
			{
				tc.gm[k][j] = z.inv(z.to_mont(PRIMES[j] % z.p));   // Montgomery form of P_j^-1
				tc.gmq[k][j] = tc.gm[k][j] * z.q;
			}
		}
	}

	// integer -> RNS register words (transformGPU.h:323-360)
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
			for (int k = 0; k < prm.K; ++k) out[(size_t)k * n + i] = (u32)(d % PRIMES[k]);
		}
	}

	// register words (first pck planes) -> integer y, then y mod N
	// (transformGPU.h:362-445: CRT over the first pck primes, carry, pack)
	void decode(const u32 * planes, mpz_t y) const
	{
		const int pck = prm.pck, lb = prm.lbase;
		const size_t nbits = (size_t)pck * lb * n, nlimbs = nbits / 64 + 2;
		std::vector<u64> out(nlimbs, 0);
		HostZp z[4] = { HostZp(PRIMES[0]), HostZp(PRIMES[1 % 14]), HostZp(PRIMES[2]), HostZp(PRIMES[3]) };
		u32 inv[4][4] = {};
		for (int i = 0; i < pck; ++i)
			for (int j = i + 1; j < pck; ++j) inv[i][j] = z[i].mul(z[i].inv(z[i].to_mont(PRIMES[j] % z[i].p)), 1);
		__int128 f = 0; size_t bit = 0;
		for (size_t i = 0; i < n; ++i)
		{
			u32 u[4];
			for (int ii = pck - 1; ii >= 0; --ii)
			{
				u32 v = planes[(size_t)ii * n + i];
				for (int j = pck - 1; j > ii; --j) v = (u32)(((u64)z[ii].sub(v, u[j]) * inv[ii][j]) % z[ii].p);
				u[ii] = v;
			}
			const int32_t i0 = (u[0] > z[0].p / 2) ? (int32_t)(u[0] - z[0].p) : (int32_t)u[0];
			__int128 D = i0;
			for (int ii = 1; ii < pck; ++ii) D = D * z[ii].p + u[ii];
			f += D;
			for (int l = 0; l < pck; ++l)
			{
				const u64 r = (u64)(f & (((__int128)1 << lb) - 1));
				const size_t li = bit / 64; const int sh = (int)(bit % 64);
				out[li] |= r << sh; if (sh != 0 && sh + lb > 64) out[li + 1] |= r >> (64 - sh);
				f >>= lb; bit += (size_t)lb;
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
	void rows(const RowJob & j0, const RowJob * j1 = nullptr, cudaStream_t s = nullptr)
	{
		RowJobs js; js.j[0] = j0; js.j[1] = j1 ? *j1 : j0;
		if (s == nullptr) { mark(); s = st; }
		CK(launch_rowpass(geo, tc, js, j1 ? 2 : 1, s));
		++launches;
	}
	void cols(const ColJob & j0, const ColJob * j1 = nullptr, cudaStream_t s = nullptr)
	{
		ColJobs js; js.j[0] = j0; js.j[1] = j1 ? *j1 : j0;
		if (s == nullptr) { mark(); s = st; }
		CK(launch_colpass(geo, tc, js, j1 ? 2 : 1, s));
		++launches;
	}
	RowJob rj(u32 * x, int mode, const u32 * w, const u32 * xp = nullptr) const
	{
		RowJob j; std::memset(&j, 0, sizeof(j)); j.x = x; j.xp = xp; j.w = w; j.mode = mode; return j;
	}
	ColJob cj_norm(const u32 * in) const
	{
		ColJob j; std::memset(&j, 0, sizeof(j)); j.in = in; j.transformed = 0; j.a = 1; return j;
	}
	ColJob cj_tr(const u32 * in, const u32 * w_in, u32 a, int nega, const u32 * sub, int lower) const
	{
		ColJob j; std::memset(&j, 0, sizeof(j));
		j.in = in; j.transformed = 1; j.w_in = w_in; j.a = a; j.nega = nega; j.sub = sub; j.lower = lower;
		return j;
	}
	static void set_fwd(ColJob & j, u32 * q_out, const u32 * wq, u32 * r_out, const u32 * wr)
	{
		j.out_fwd[0] = q_out; j.w_out[0] = q_out ? wq : nullptr;
		j.out_fwd[1] = r_out; j.w_out[1] = r_out ? wr : nullptr;
	}

	// full forward transform of a normal-form register in one or two domains
	void full_forward(const u32 * src, u32 * dq, u32 * dr)
	{
		ColJob j = cj_norm(src); set_fwd(j, dq, b(WQ), dr, b(WR)); cols(j);
		if (dq && dr) { RowJob a = rj(dq, ROW_FWD_ONLY, b(WQ)), c = rj(dr, ROW_FWD_ONLY, b(WR)); rows(a, &c); }
		else if (dq) rows(rj(dq, ROW_FWD_ONLY, b(WQ)));
		else rows(rj(dr, ROW_FWD_ONLY, b(WR)));
	}

	// reduceMMGW tail (transformGPU.h:523-538): m' = T_R Ninv mod R, +2,
	// r' = m' N - T_Q mod Q.  AR1 holds the first forward levels of T_R.
	void reduce_tail(const u32 * tq, u32 * out, bool want_prefwd, bool join_q = false)
	{
		rows(rj(b(AR1), ROW_MUL, b(WR), b(NIR)));
		ColJob j1 = cj_tr(b(AR1), b(WR), 1, 0, nullptr, LOWER_R_ADD2); set_fwd(j1, b(AQ1), b(WQ), nullptr, nullptr); cols(j1);
		rows(rj(b(AQ1), ROW_MUL, b(WQ), b(NQ)));
		if (join_q) CK(cudaStreamWaitEvent(st, ev_q, 0));
		ColJob j2 = cj_tr(b(AQ1), b(WQ), 1, 1, tq, LOWER_Q); j2.out_norm = out;
		j2.sub_big = (tq == b(TQ)) ? 1 : 0;     // T_Q of first_product holds exact coefficient values
		if (want_prefwd) set_fwd(j2, b(AQ0), b(WQ), b(AR0), b(WR));
		cols(j2);
	}

	// First product of squareMMGW / mulMMGW (transformGPU.h:540-568):
	// T_Q = carry(x y mod Q) into TQ and the first forward levels of
	// carry(x y mod R) into AR1.  AQ0/AR0 hold the first forward levels of x;
	// xq/xr the full forward images of y (nullptr: y = x, square).  With
	// overlap, the Q chain runs on st2 (T_Q is only needed by the final
	// carry-sub) and reduce_tail joins it.  A non-null `mult` is a device word
	// read in place of `a` (graph replays).
	void first_product(u32 a, const u32 * xq, const u32 * xr, const u32 * mult = nullptr)
	{
		RowJob rq = rj(b(AQ0), xq ? ROW_MUL : ROW_SQUARE, b(WQ), xq), rr = rj(b(AR0), xr ? ROW_MUL : ROW_SQUARE, b(WR), xr);
		ColJob jq = cj_tr(b(AQ0), b(WQ), a, 1, nullptr, LOWER_NONE); jq.out_norm = b(TQ); jq.out_big = 1; jq.mult = mult;
		ColJob jr = cj_tr(b(AR0), b(WR), a, 0, nullptr, LOWER_NONE); set_fwd(jr, nullptr, nullptr, b(AR1), b(WR)); jr.mult = mult;
		if (overlap)
		{
			CK(cudaEventRecord(ev_fork, st));
			CK(cudaStreamWaitEvent(st2, ev_fork, 0));
			rows(rq, nullptr, st2);
			cols(jq, nullptr, st2);
			CK(cudaEventRecord(ev_q, st2));
			rows(rr);
			cols(jr);
		}
		else if (split)
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

	// squareMMGW (transformGPU.h:556-568)
	void square_mul(u32 a)
	{
		if (!prefwd) { ColJob j = cj_norm(b(REG0)); set_fwd(j, b(AQ0), b(WQ), b(AR0), b(WR)); cols(j); }
		first_product(a, nullptr, nullptr);
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
					first_product(1, nullptr, nullptr, d_mult + s);
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
		if (!prefwd) { ColJob j = cj_norm(b(REG0)); set_fwd(j, b(AQ0), b(WQ), b(AR0), b(WR)); cols(j); }
		const int hi = mult_i;
		CK(cudaEventSynchronize(mult_done[hi]));
		std::memcpy(h_mult[hi], mults, G * sizeof(u32));
		CK(cudaMemcpyAsync(d_mult, h_mult[hi], G * sizeof(u32), cudaMemcpyHostToDevice, st));
		CK(cudaEventRecord(mult_done[hi], st));
		mult_i ^= 1;
		CK(cudaGraphLaunch(gexec, st));
		launches += graph_kernels;
		prefwd = true;
	}

	// the split and the launch constants that describe it, always together
	void use_geometry(const Geometry & g)
	{
		geo = g;
		tc.R = g.R; tc.H = g.H; tc.LA = g.LA; tc.LB = g.LB;
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
		{ ColJob j = cj_norm(b(dst)); set_fwd(j, b(AQ0), b(WQ), b(AR0), b(WR)); cols(j); }
		prefwd = false;
		first_product(1, b(OPQ), b(OPR));
		reduce_tail(b(TQ), b(dst), dst == REG0, overlap);
		prefwd = (dst == REG0);
	}

	// conversion out of MMGW form into TMP (transformGPU.h:576-586)
	void reduce_copy(int src)
	{
		ColJob j = cj_norm(b(src)); set_fwd(j, nullptr, nullptr, b(AR1), b(WR)); cols(j);
		reduce_tail(b(src), b(TMP), false);
	}

	void copy(int dst, int src)
	{
		if (dst == src) return;
		CK(cudaMemcpyAsync(b(dst), b(src), (size_t)prm.K * n * 4, cudaMemcpyDeviceToDevice, st));
		if (dst == REG0) prefwd = false;
	}

	void upload(int buf, const u32 * src)
	{
		CK(cudaMemcpyAsync(b(buf), src, (size_t)prm.K * n * 4, cudaMemcpyHostToDevice, st));
		CK(cudaStreamSynchronize(st));
	}
	void download(int buf, u32 * dst, size_t planes)
	{
		CK(cudaMemcpyAsync(dst, b(buf), planes * n * 4, cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
	}

	void get(int src, mpz_t z)
	{
		reduce_copy(src);
		host.resize((size_t)prm.K * n);
		download(TMP, host.data(), (size_t)prm.pck);
		decode(host.data(), z);
	}

	// host part of the set-up: parameters, geometry, R, N^-1 mod R, constants,
	// and the register words of N, N^-1 and the MMGW form of 1
	struct Prepared
	{
		std::vector<u32> wN, wNinv, wOne;
	};

	void prepare(const mpz_t Nin, int32_t a, const ab_params * forced, Prepared & pp)
	{
		mpz_set(N, Nin);
		prm = forced ? *forced : select_params(N, a);
		if (prm.K < 2 || prm.K > 5 || (size_t)prm.pck != get_s((size_t)prm.K) || prm.lbase < 2 || prm.lbase > 31)
			throw ab_error(AB_E_ARG, "invalid transform parameters");
		if (!make_geometry(prm.ln, 0, geo)) throw ab_error(AB_E_UNSUPPORTED, "NTT length 2^" + std::to_string(prm.ln) + " is not supported (6 <= ln <= 20)");
		n = (size_t)1 << prm.ln;
		mpz_t R, Ninv; mpz_inits(R, Ninv, nullptr);
		if (!compute_R_Ninv(N, prm, R, Ninv, factor)) { failed = true; mpz_clears(R, Ninv, nullptr); return; }
		build_consts();
		const size_t words = (size_t)prm.K * n;
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
		CK(cudaMalloc(&dmem, (size_t)NBUF * prm.K * n * 4));
		CK(cudaMemsetAsync(dmem, 0, (size_t)NBUF * prm.K * n * 4, st));
		for (int i = 0; i < NBUF; ++i) bufp[i] = dmem + (size_t)i * prm.K * n;

		host.assign((size_t)prm.K * n, 0);
		std::vector<u32> wr((size_t)prm.K * n), wq((size_t)prm.K * n);
		for (int k = 0; k < prm.K; ++k) { make_roots(&wr[(size_t)k * n], prm.ln, k, false); make_roots(&wq[(size_t)k * n], prm.ln, k, true); }
		upload(WR, wr.data()); upload(WQ, wq.data());
		setup_device(pp);
	}
};

// ============================================================ batches
// A size class (K, pck, ln) of `cap` candidates with stacked buffers: buffer
// type i of slot s is at base[i] + s * words.  Each loaded slot is exposed as
// an ab_transform view (set1 / copy / mul / get work unchanged on it); the
// squarings of all slots run together (grid.z = slot) from a captured CUDA
// graph whose per-step, per-slot multipliers are uploaded before each launch.
struct ab_batch
{
	int device = 0;
	cudaStream_t st = nullptr;
	ab_params cls{};
	Geometry geo{};
	TConst tc{};
	size_t n = 0, words = 0;
	int cap = 0, max_steps = 0;
	u32 * mem = nullptr;
	u32 * base[ab_transform::NBUF] = {};
	CandConst * d_cand = nullptr;
	std::vector<CandConst> h_cand;
	u32 * d_ctrl = nullptr;            // per step: mult[cap] | act[cap] | snap[cap]
	u32 * h_ctrl[2] = {};              // page-locked staging, alternating between launches
	cudaEvent_t ctrl_done[2] = {};     // the upload out of h_ctrl[i] has completed
	int ctrl_i = 0;
	std::vector<ab_transform *> views;
	cudaGraphExec_t gexec = nullptr;
	int g_steps = 0;
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
		if (st) cudaStreamDestroy(st);
	}

	u32 * ctrl(int step, int part) const { return d_ctrl + ((size_t)step * 3 + part) * cap; }

	void rows(const RowJob & j0, const RowJob * j1 = nullptr)
	{
		RowJobs js; js.j[0] = j0; js.j[1] = j1 ? *j1 : j0;
		CK(launch_rowpass(geo, tc, js, j1 ? 2 : 1, st, zl));
	}
	void cols(const ColJob & j0, const ColJob * j1 = nullptr)
	{
		ColJobs js; js.j[0] = j0; js.j[1] = j1 ? *j1 : j0;
		CK(launch_colpass(geo, tc, js, j1 ? 2 : 1, st, zl));
	}
	RowJob rj(u32 * x, int mode, const u32 * w, const u32 * xp, const u32 * act) const
	{
		RowJob j; std::memset(&j, 0, sizeof(j));
		j.x = x; j.xp = xp; j.w = w; j.mode = mode; j.stride = words; j.active = act;
		return j;
	}
	ColJob cj(const u32 * in, bool tr, const u32 * w_in, const u32 * mult, int nega, const u32 * sub, int lower) const
	{
		ColJob j; std::memset(&j, 0, sizeof(j));
		j.in = in; j.transformed = tr ? 1 : 0; j.w_in = w_in; j.a = 1; j.mult = mult; j.nega = nega; j.sub = sub;
		j.lower = lower; j.stride = words; j.cand = d_cand;
		return j;
	}

	// squareMMGW (transformGPU.h:556-568) for every slot, `steps` times
	void record_steps(int steps)
	{
		using T = ab_transform;
		u32 * const aq0 = base[T::AQ0], * const ar0 = base[T::AR0], * const aq1 = base[T::AQ1], * const ar1 = base[T::AR1];
		const u32 * wq = base[T::WQ], * wr = base[T::WR];
		{
			ColJob j = cj(base[T::REG0], false, nullptr, ctrl(0, 1), 0, nullptr, LOWER_NONE);
			j.out_fwd[0] = aq0; j.w_out[0] = wq; j.out_fwd[1] = ar0; j.w_out[1] = wr;
			cols(j);
		}
		for (int s = 0; s < steps; ++s)
		{
			const u32 * mult = ctrl(s, 0), * act = ctrl(s, 1), * snap = ctrl(s, 2);
			RowJob rq = rj(aq0, ROW_SQUARE, wq, nullptr, act), rr = rj(ar0, ROW_SQUARE, wr, nullptr, act);
			rows(rq, &rr);
			ColJob jq = cj(aq0, true, wq, mult, 1, nullptr, LOWER_NONE); jq.out_norm = base[T::TQ]; jq.out_big = 1;
			ColJob jr = cj(ar0, true, wr, mult, 0, nullptr, LOWER_NONE); jr.out_fwd[1] = ar1; jr.w_out[1] = wr;
			cols(jq, &jr);
			rows(rj(ar1, ROW_MUL, wr, base[T::NIR], act));
			ColJob j1 = cj(ar1, true, wr, act, 0, nullptr, LOWER_R_ADD2); j1.out_fwd[0] = aq1; j1.w_out[0] = wq;
			cols(j1);
			rows(rj(aq1, ROW_MUL, wq, base[T::NQ], act));
			ColJob j2 = cj(aq1, true, wq, act, 1, base[T::TQ], LOWER_Q); j2.sub_big = 1;
			j2.out_norm = base[T::REG0];
			j2.out_fwd[0] = aq0; j2.w_out[0] = wq; j2.out_fwd[1] = ar0; j2.w_out[1] = wr;
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
		// per prime k: plane k of Reg0 then plane k of Reg1 (transformGPU.h:626-641)
		for (size_t k = 0; k < K; ++k)
		{
			CK(cudaMemcpyAsync(o + 2 + 2 * k * n, h->b(ab_transform::REG0) + k * n, n * 4, cudaMemcpyDeviceToHost, h->st));
			CK(cudaMemcpyAsync(o + 2 + 2 * k * n + n, h->b(ab_transform::REG1) + k * n, n * 4, cudaMemcpyDeviceToHost, h->st));
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
		for (size_t k = 0; k < K; ++k)
		{
			CK(cudaMemcpyAsync(h->b(ab_transform::REG0) + k * n, in + 2 + 2 * k * n, n * 4, cudaMemcpyHostToDevice, h->st));
			CK(cudaMemcpyAsync(h->b(ab_transform::REG1) + k * n, in + 2 + 2 * k * n + n, n * 4, cudaMemcpyHostToDevice, h->st));
		}
		CK(cudaStreamSynchronize(h->st));
		h->prefwd = false;
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
		h->download((int)reg, out, (size_t)h->prm.K);
	});
}

int ab_write_register(ab_transform * h, size_t reg, const uint32_t * in, size_t nwords)
{
	return guarded([&] {
		need_ready(h);
		if (!valid_reg(reg) || in == nullptr || nwords != (size_t)h->prm.K * h->n) throw ab_error(AB_E_ARG, "bad arguments");
		h->upload((int)reg, in);
		if (reg == 0) h->prefwd = false;
	});
}

int ab_synchronize(ab_transform * h)
{
	return guarded([&] { if (h == nullptr) throw ab_error(AB_E_ARG, "null handle"); if (h->st) CK(cudaStreamSynchronize(h->st)); });
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
		const size_t words = (size_t)h->prm.K * h->n;
		if (words > AB_NOALLOC_MAX_WORDS)
			throw ab_error(AB_E_CAPACITY, "ab_square_mul_noalloc: K*n = " + std::to_string(words) +
				" words exceeds the static scratch limit of " + std::to_string(AB_NOALLOC_MAX_WORDS) + " words per register");
		u32 * const s = (h->noalloc != nullptr) ? h->noalloc : noalloc_scratch(h->device);
		u32 * const aq0 = s, * const ar0 = s + AB_NOALLOC_MAX_WORDS, * const aq1 = s + 2 * AB_NOALLOC_MAX_WORDS;
		u32 * const ar1 = s + 3 * AB_NOALLOC_MAX_WORDS, * const tq = s + 4 * AB_NOALLOC_MAX_WORDS;
		using T = ab_transform;
		const u32 * wq = h->b(T::WQ), * wr = h->b(T::WR);
		// squareMMGW (transformGPU.h:556-568) with every intermediate in the
		// static scratch: each scratch word is written before it is read
		// within the call, so nothing needs clearing between calls
		ColJob j0 = h->cj_norm(reg); T::set_fwd(j0, aq0, wq, ar0, wr); h->cols(j0);
		RowJob rq = h->rj(aq0, ROW_SQUARE, wq), rr = h->rj(ar0, ROW_SQUARE, wr);
		h->rows(rq, &rr);
		ColJob jq = h->cj_tr(aq0, wq, (u32)a, 1, nullptr, LOWER_NONE); jq.out_norm = tq;
		ColJob jr = h->cj_tr(ar0, wr, (u32)a, 0, nullptr, LOWER_NONE); T::set_fwd(jr, nullptr, nullptr, ar1, wr);
		h->cols(jq, &jr);
		h->rows(h->rj(ar1, ROW_MUL, wr, h->b(T::NIR)));
		ColJob j1 = h->cj_tr(ar1, wr, 1, 0, nullptr, LOWER_R_ADD2); T::set_fwd(j1, aq1, wq, nullptr, nullptr); h->cols(j1);
		h->rows(h->rj(aq1, ROW_MUL, wq, h->b(T::NQ)));
		ColJob j2 = h->cj_tr(aq1, wq, 1, 1, tq, LOWER_Q); j2.out_norm = reg; h->cols(j2);
	});
}

int ab_diag_forward(ab_transform * h, int domain, const uint32_t * in, uint32_t * out)
{
	return guarded([&] {
		need_ready(h);
		h->upload(ab_transform::TMP, in);
		if (domain) h->full_forward(h->b(ab_transform::TMP), h->b(ab_transform::AQ1), nullptr);
		else h->full_forward(h->b(ab_transform::TMP), nullptr, h->b(ab_transform::AQ1));
		h->download(ab_transform::AQ1, out, (size_t)h->prm.K);
	});
}

int ab_diag_product(ab_transform * h, int domain, const uint32_t * in, const uint32_t * xp, uint32_t a,
	const uint32_t * sub, int lower_mode, uint32_t * out)
{
	return guarded([&] {
		need_ready(h);
		using T = ab_transform;
		const u32 * w = h->b(domain ? T::WQ : T::WR);
		h->upload(T::TMP, in);
		if (xp) h->upload(T::OPQ, xp);
		if (sub) h->upload(T::OPR, sub);
		ColJob j = h->cj_norm(h->b(T::TMP));
		if (domain) T::set_fwd(j, h->b(T::AQ1), w, nullptr, nullptr); else T::set_fwd(j, nullptr, nullptr, h->b(T::AQ1), w);
		h->cols(j);
		h->rows(h->rj(h->b(T::AQ1), xp ? ROW_MUL : ROW_SQUARE, w, xp ? h->b(T::OPQ) : nullptr));
		ColJob c = h->cj_tr(h->b(T::AQ1), w, a, domain ? 1 : 0, sub ? h->b(T::OPR) : nullptr, lower_mode);
		c.out_norm = h->b(T::TMP);
		h->cols(c);
		h->download(T::TMP, out, (size_t)h->prm.K);
		h->prefwd = false;
	});
}


size_t ab_batch_slot_bytes(const ab_params * cls)
{
	if (cls == nullptr) return 0;
	return (size_t)(ab_transform::WR) * cls->K * ((size_t)1 << cls->ln) * 4;
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
		b->n = (size_t)1 << cls->ln; b->words = (size_t)cls->K * b->n;
		CK(cudaSetDevice(device));
		CK(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
		const size_t per = (size_t)ab_transform::WR;          // per-slot buffer types
		CK(cudaMalloc(&b->mem, (per * capacity + 2) * b->words * 4));
		CK(cudaMemsetAsync(b->mem, 0, (per * capacity + 2) * b->words * 4, b->st));
		for (size_t i = 0; i < per; ++i) b->base[i] = b->mem + i * capacity * b->words;
		b->base[ab_transform::WR] = b->mem + per * capacity * b->words;
		b->base[ab_transform::WQ] = b->base[ab_transform::WR] + b->words;
		std::vector<u32> wr(b->words), wq(b->words);
		for (int k = 0; k < cls->K; ++k) { make_roots(&wr[(size_t)k * b->n], cls->ln, k, false); make_roots(&wq[(size_t)k * b->n], cls->ln, k, true); }
		CK(cudaMemcpyAsync(b->base[ab_transform::WR], wr.data(), b->words * 4, cudaMemcpyHostToDevice, b->st));
		CK(cudaMemcpyAsync(b->base[ab_transform::WQ], wq.data(), b->words * 4, cudaMemcpyHostToDevice, b->st));
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
		b->views.assign(capacity, nullptr);
		// TConst of the class (digit constants come from d_cand)
		ab_transform probe_t;
		probe_t.prm = *cls; probe_t.prm.lbase = 17; probe_t.n = b->n; probe_t.geo = b->geo;
		probe_t.build_consts();
		b->tc = probe_t.tc;
		probe_t.view = true;
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

// Device part: the slot's buffers, the transforms of N and N^-1, the constants
// of its digit size; the view then owns the slot.
void batch_install(ab_batch * b, int slot, std::unique_ptr<ab_transform> & vp, const ab_transform::Prepared & pp)
{
	ab_transform * v = vp.get();
	if (!v->failed && (v->prm.K != b->cls.K || v->prm.pck != b->cls.pck || v->prm.ln != b->cls.ln))
		throw ab_error(AB_E_ARG, "N does not belong to this size class");
	delete b->views[slot];
	b->views[slot] = nullptr;
	v->device = b->device; v->st = b->st; v->overlap = false;
	v->noalloc = noalloc_scratch(b->device);
	v->use_geometry(b->geo);             // the batch's split, which the autotuner may have changed
	for (int i = 0; i < ab_transform::WR; ++i) v->bufp[i] = b->base[i] + (size_t)slot * b->words;
	v->bufp[ab_transform::WR] = b->base[ab_transform::WR];
	v->bufp[ab_transform::WQ] = b->base[ab_transform::WQ];
	if (!v->failed)
	{
		v->host.assign(b->words, 0);
		v->setup_device(pp);
		CandConst & c = b->h_cand[slot];
		c.lbase = v->prm.lbase;
		for (int k = 0; k < AB_MAXK; ++k) { c.rbase[k] = v->tc.rbase[k]; c.rbase_pck[k] = v->tc.rbase_pck[k]; }
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
		v->prm = s->prm; v->n = s->n; v->geo = s->geo; v->tc = s->tc; v->failed = s->failed;
		v->device = b->device; v->st = b->st; v->overlap = false;
		v->noalloc = s->noalloc;
		v->host.assign(b->words, 0);
		for (int i = 0; i < ab_transform::WR; ++i) v->bufp[i] = b->base[i] + (size_t)dst * b->words;
		v->bufp[ab_transform::WR] = b->base[ab_transform::WR];
		v->bufp[ab_transform::WQ] = b->base[ab_transform::WQ];
		for (int i = 0; i < ab_transform::WR; ++i)
			CK(cudaMemcpyAsync(v->bufp[i], s->bufp[i], b->words * 4, cudaMemcpyDeviceToDevice, b->st));
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
			CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
			try { b->record_steps(steps); }
			catch (...) { cudaStreamEndCapture(b->st, &g); if (g) cudaGraphDestroy(g); throw; }
			CK(cudaStreamEndCapture(b->st, &g));
			const cudaError_t e = cudaGraphInstantiate(&b->gexec, g, 0);
			cudaGraphDestroy(g);
			CK(e);
			b->g_steps = steps;
		}
		CK(cudaGraphLaunch(b->gexec, b->st));
		b->launches += 1 + 6 * (uint64_t)steps;       // kernels of the graph
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
		b->tc.R = g.R; b->tc.H = g.H; b->tc.LA = g.LA; b->tc.LB = g.LB;
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
