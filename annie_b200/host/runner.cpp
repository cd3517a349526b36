// Continuous-batching PRP runner (include/annie_b200_batch.h).
//
// Each test runs the program of the reference driver (src/annie.h:217-430):
//   MAIN    square_mul over the bits of E from the top, Gerbicz-Li product
//           d *= Reg0 at every block boundary (kept by the batch graph, then
//           multiplied in by ab_batch_gl_mul);
//   EULER   one more squaring for the Euler test (a^(N-1));
//   GL_HI   Reg0 = 1, square_mul over the bits of res above B;
//   GL_LO   Reg0 *= d, then B square_mul with the low bits of res;
//   check   Reg0 ?= d(t+1) (kept in Reg2).
// With gl_check_blocks > 0, MAIN stops every gl_check_blocks blocks for a
// periodic check (not in the reference, which checks only at the end):
//   CHK_HI, CHK_LO   the same power a^C d_prev^(2^B) with C the chunk sum of
//                    E >> i, then Reg0 ?= d(t); the test's (Reg0, Reg1) were
//                    saved before and are restored after; on a mismatch the
//                    test rolls back to its last verified state.
// Squarings of all admitted tests run together, one graph launch per chunk
// and size class; the host steps between phases use the slot's transform.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "gmp.h"
#include "../../include/annie_b200_batch.h"

namespace
{
int ilog2_32(uint32_t n) { return (n == 0) ? -1 : (31 - __builtin_clz(n)); }

int gl_block_size(size_t size)
{
	const size_t L = size_t(2) << (ilog2_32(uint32_t(size)) / 2);
	return int((size - 1) / L) + 1;
}

void chunk_sum(mpz_t res, const mpz_t e_in, int B)
{
	mpz_t e, t; mpz_init_set(e, e_in); mpz_init(t);
	mpz_set_ui(res, 0);
	while (mpz_sgn(e) != 0)
	{
		mpz_fdiv_r_2exp(t, e, (mp_bitcnt_t)B);
		mpz_add(res, res, t);
		mpz_fdiv_q_2exp(e, e, (mp_bitcnt_t)B);
	}
	mpz_clears(e, t, nullptr);
}

struct rt_error : std::runtime_error { using std::runtime_error::runtime_error; };

void ck(int rc)
{
	if (rc != AB_OK) throw rt_error(ab_last_error());
}

enum Phase { MAIN, EULER, GL_HI, GL_LO, CHK_HI, CHK_LO, DONE };

struct Job
{
	uint64_t tag = 0;
	mpz_t N, E, res, chk;
	int euler = 0;
	int32_t a = 2;
	int B = 0;
	long i = 0;           // next bit of the current phase's exponent (counting down)
	Phase ph = MAIN;
	ab_prp_result r{};
	std::vector<uint64_t> limbs;

	// periodic Gerbicz-Li checks: blocks since the last verified state, the
	// bit at which the running check was taken, the verified state (payload of
	// Reg0 and Reg1) and the bit below which it resumes, the state saved while
	// a check runs
	int blocks = 0, fails_in_row = 0;
	long chk_bit = -1, vi = -1;
	std::vector<uint8_t> vsnap, stash;
	bool injected = false;

	Job() { mpz_inits(N, E, res, chk, nullptr); }
	~Job() { mpz_clears(N, E, res, chk, nullptr); }

	// bit that the next squaring of the current phase uses, and its multiplier
	uint32_t mult_at(long bit) const
	{
		if (ph == MAIN) return mpz_tstbit(E, (mp_bitcnt_t)bit) ? (uint32_t)a : 1u;
		if (ph == EULER) return 1u;
		if (ph == CHK_HI || ph == CHK_LO) return mpz_tstbit(chk, (mp_bitcnt_t)bit) ? (uint32_t)a : 1u;
		return mpz_tstbit(res, (mp_bitcnt_t)bit) ? (uint32_t)a : 1u;   // GL_HI / GL_LO
	}
	long low_bit() const { return (ph == GL_HI || ph == CHK_HI) ? B : 0; }
	long remaining() const { return (ph == DONE) ? 0 : i - low_bit() + 1; }
};

struct Class
{
	ab_params cls{};
	ab_batch * b = nullptr;
	int cap = 0;
	std::vector<Job *> slots;
	std::vector<uint32_t> mult;
	std::vector<uint8_t> snap;
	std::vector<int> count;
	bool tuned = false;
	size_t bytes = 0;                  // device memory of the batch
	uint64_t last_used = 0;            // runner tick of the last chunk or admission
};

std::string hex64(uint64_t u)
{
	char b[32];
	std::snprintf(b, sizeof(b), "%016llX", (unsigned long long)u);
	return b;
}
}

struct ab_runner
{
	ab_runner_options o{};
	std::deque<Job *> queue;
	std::deque<Job *> done;
	std::vector<std::unique_ptr<Class>> classes;
	size_t used = 0;
	uint64_t squarings = 0;
	uint64_t tick = 0;                 // advance() calls

	~ab_runner()
	{
		for (auto & c : classes)
		{
			for (Job * j : c->slots) delete j;
			ab_batch_destroy(c->b);
		}
		for (Job * j : queue) delete j;
		for (Job * j : done) delete j;
	}

	void finish(Job * j, int status, const char * msg)
	{
		j->r.status = status;
		std::snprintf(j->r.message, sizeof(j->r.message), "%s", msg);
		j->ph = DONE;
		done.push_back(j);
	}

	// host part of admission: trivial cases, base, parameters; returns false
	// when the job was decided without a transform
	bool classify(Job * j, ab_params & p)
	{
		const mpz_srcptr n = j->N;
		if (mpz_sizeinbase(n, 2) <= 50 && mpz_cmp_ui(n, 999999999999999ul) <= 0)
		{
			j->r.decided_early = 1;
			const int pp = mpz_probab_prime_p(n, 20);
			j->r.is_prp = pp != 0;
			finish(j, 0, (pp != 0) ? "N is a probable prime." : "N is composite.");
			return false;
		}
		if (mpz_even_p(n)) { j->r.decided_early = 1; finish(j, 0, "N is even."); return false; }
		if (j->euler)
		{
			int32_t a = 2;
			while (mpz_si_kronecker(a, n) != -1)
			{
				++a;
				const int32_t s = (int32_t)std::lround(std::sqrt(double(a)));
				if (s * s == a) ++a;
			}
			j->a = a;
		}
		j->r.base = j->a;
		ck(ab_probe(j->limbs.data(), j->limbs.size(), j->a, nullptr, &p, nullptr));
		return true;
	}

	// frees batches that hold no test, least recently used first, until `need`
	// more bytes fit the budget, so that tests of other size classes can be
	// admitted once the budget is spent (a long-running server sees many sizes
	// over time); the batches that stay keep their graphs and tuned split
	void reclaim(size_t need)
	{
		while (used + need > o.hbm_budget_bytes)
		{
			auto victim = classes.end();
			for (auto it = classes.begin(); it != classes.end(); ++it)
			{
				const Class & c = **it;
				if (!std::all_of(c.slots.begin(), c.slots.end(), [](Job * j) { return j == nullptr; })) continue;
				if (victim == classes.end() || c.last_used < (*victim)->last_used) victim = it;
			}
			if (victim == classes.end()) return;
			ab_batch_destroy((*victim)->b);
			used -= (*victim)->bytes;
			classes.erase(victim);
		}
	}

	Class * class_for(const ab_params & p, bool create)
	{
		for (auto & c : classes)
			if (c->cls.K == p.K && c->cls.pck == p.pck && c->cls.ln == p.ln)
				for (Job * s : c->slots) if (s == nullptr) { c->last_used = tick; return c.get(); }
		if (!create) return nullptr;
		ab_params cls = p; cls.lbase = 0;
		const size_t per = ab_batch_slot_bytes(&cls);
		if (used + per > o.hbm_budget_bytes) reclaim(per);
		if (used + per > o.hbm_budget_bytes) return nullptr;
		const int cap = (int)std::min<size_t>((size_t)o.max_slots_per_class, (o.hbm_budget_bytes - used) / per);
		if (cap < 1) return nullptr;
		auto c = std::make_unique<Class>();
		c->cls = cls; c->cap = cap;
		ck(ab_batch_create(o.device, &cls, cap, o.chunk, &c->b));
		c->slots.assign(cap, nullptr);
		c->mult.assign((size_t)o.chunk * cap, 0);
		c->snap.assign((size_t)o.chunk * cap, 0);
		c->bytes = per * cap;
		c->last_used = tick;
		used += c->bytes;
		classes.push_back(std::move(c));
		return classes.back().get();
	}

	// Admission: classify queued tests, reserve a slot of their size class
	// (creating the class within the HBM budget), then load each class's new
	// slots together (host set-up on threads) and start their tests.
	void admit()
	{
		std::deque<Job *> later;
		struct Pending { Class * c; int slot; Job * j; };
		std::vector<Pending> pend;
		while (!queue.empty())
		{
			Job * j = queue.front(); queue.pop_front();
			ab_params p{};
			if (j->ph == MAIN && j->B == 0)
			{
				if (!classify(j, p)) continue;
				j->r.K = p.K; j->r.pck = p.pck; j->r.ln = p.ln; j->r.lbase = p.lbase;
				j->B = -1;     // classified
			}
			else { p.K = j->r.K; p.pck = j->r.pck; p.ln = j->r.ln; p.lbase = j->r.lbase; }
			Class * c = class_for(p, true);
			if (c == nullptr) { later.push_back(j); continue; }
			const int slot = (int)(std::find(c->slots.begin(), c->slots.end(), nullptr) - c->slots.begin());
			c->slots[slot] = j;                   // reserved
			pend.push_back({c, slot, j});
		}
		queue.swap(later);

		std::vector<Class *> order;
		for (const Pending & q : pend) if (std::find(order.begin(), order.end(), q.c) == order.end()) order.push_back(q.c);
		for (Class * c : order)
		{
			std::vector<Pending> mine;
			for (const Pending & q : pend) if (q.c == c) mine.push_back(q);
			const int cnt = (int)mine.size();
			std::vector<int> slots(cnt), failed(cnt, 0);
			std::vector<const uint64_t *> nl(cnt);
			std::vector<size_t> nn(cnt);
			std::vector<int32_t> aa(cnt);
			for (int i = 0; i < cnt; ++i)
			{
				slots[i] = mine[i].slot; nl[i] = mine[i].j->limbs.data(); nn[i] = mine[i].j->limbs.size(); aa[i] = mine[i].j->a;
			}
			ck(ab_batch_load_many(c->b, cnt, slots.data(), nl.data(), nn.data(), aa.data(), failed.data()));
			for (int i = 0; i < cnt; ++i)
			{
				Job * j = mine[i].j;
				const int slot = mine[i].slot;
				ab_transform * v = ab_batch_slot(c->b, slot);
				if (failed[i])
				{
					std::vector<uint64_t> f(j->limbs.size() + 2);
					size_t fc = 0;
					ck(ab_get_factor(v, f.data(), f.size(), &fc));
					ab_batch_release(c->b, slot);
					c->slots[slot] = nullptr;
					mpz_t z; mpz_init(z); mpz_import(z, fc, -1, 8, 0, 0, f.data());
					char * s = mpz_get_str(nullptr, 10, z);
					char msg[256]; std::snprintf(msg, sizeof(msg), "%.200s divides N.", s);
					free(s); mpz_clear(z);
					j->r.decided_early = 1;
					finish(j, 0, msg);
					continue;
				}
				ck(ab_set1(v));
				ck(ab_copy(v, 1, 0));
				if (!c->tuned)
				{
					int lb = 0;
					if (o.autotune) ck(ab_batch_autotune(c->b, slot, o.chunk, &lb));
					c->tuned = true;
				}
				mpz_sub_ui(j->E, j->N, 1);
				if (j->euler) mpz_fdiv_q_2exp(j->E, j->E, 1);
				j->B = gl_block_size(mpz_sizeinbase(j->E, 2));
				j->r.gl_block = j->B;
				j->i = (long)mpz_sizeinbase(j->E, 2) - 1;
				j->ph = MAIN;
				if (o.gl_check_blocks > 0) { j->vsnap = payload(v); j->vi = j->i + 1; }
			}
		}
	}

	static std::vector<uint8_t> payload(ab_transform * v)
	{
		std::vector<uint8_t> buf(ab_checkpoint_size(v));
		size_t w = 0;
		ck(ab_save_checkpoint(v, buf.data(), buf.size(), &w));
		return buf;
	}

	// a periodic check at the block boundary just passed (bit chk_bit): Reg2 =
	// d before this block's factor, Reg1 = d now; save (Reg0, Reg1), then
	// compute a^C Reg2^(2^B) in Reg0 over the CHK phases
	void start_check(ab_transform * v, Job * j)
	{
		j->stash = payload(v);
		mpz_t e; mpz_init(e);
		mpz_fdiv_q_2exp(e, j->E, (mp_bitcnt_t)j->chk_bit);
		chunk_sum(j->chk, e, j->B);
		mpz_clear(e);
		ck(ab_set1(v));
		++j->r.gl_checks;
		j->ph = CHK_HI;
		j->i = (long)mpz_sizeinbase(j->chk, 2) - 1;
		if (j->i < j->B) { ck(ab_mul(v, 0, 2)); j->ph = CHK_LO; j->i = j->B - 1; }
	}

	// the check's power is in Reg0: compare with d(t) in Reg1, then resume at
	// the checked state or roll back to the last verified one
	void end_check(ab_transform * v, Job * j, std::vector<uint64_t> & buf)
	{
		size_t cnt = 0;
		mpz_t z0, z1; mpz_inits(z0, z1, nullptr);
		ck(ab_get(v, 0, buf.data(), buf.size(), &cnt)); mpz_import(z0, cnt, -1, 8, 0, 0, buf.data());
		ck(ab_get(v, 1, buf.data(), buf.size(), &cnt)); mpz_import(z1, cnt, -1, 8, 0, 0, buf.data());
		const bool ok = mpz_cmp(z0, z1) == 0;
		mpz_clears(z0, z1, nullptr);
		j->blocks = 0;
		j->ph = MAIN;
		if (ok)
		{
			ck(ab_read_checkpoint(v, j->stash.data(), j->stash.size()));
			j->vsnap.swap(j->stash);
			j->vi = j->chk_bit;
			j->i = j->chk_bit - 1;
			j->fails_in_row = 0;
		}
		else
		{
			ck(ab_read_checkpoint(v, j->vsnap.data(), j->vsnap.size()));
			j->i = j->vi - 1;
			++j->r.gl_failures;
			++j->r.rollbacks;
			++j->fails_in_row;
		}
		j->stash.clear();
	}

	// host steps at the end of a phase (src/annie.h:343-403)
	void next_phase(Class & c, int slot, Job * j)
	{
		ab_transform * v = ab_batch_slot(c.b, slot);
		std::vector<uint64_t> buf(j->limbs.size() + 2);
		if (j->ph == CHK_HI) { ck(ab_mul(v, 0, 2)); j->ph = CHK_LO; j->i = j->B - 1; return; }
		if (j->ph == CHK_LO) { end_check(v, j, buf); return; }
		size_t cnt = 0;
		mpz_t z; mpz_init(z);
		auto get = [&](size_t reg) {
			ck(ab_get(v, reg, buf.data(), buf.size(), &cnt));
			mpz_import(z, cnt, -1, 8, 0, 0, buf.data());
		};
		if (j->ph == MAIN)
		{
			ck(ab_copy(v, 2, 0));
			ck(ab_mul(v, 2, 1));                       // d(t+1)
			get(0);
			if (j->euler)
			{
				mpz_add_ui(z, z, 1);
				if (mpz_cmp(z, j->N) >= 0) mpz_sub(z, z, j->N);
				j->r.is_prp = (mpz_sgn(z) == 0);
				j->ph = EULER; j->i = 0;
				mpz_clear(z);
				return;
			}
			mpz_sub_ui(z, z, 1);
			j->r.is_prp = (mpz_sgn(z) == 0);
		}
		if (j->ph == MAIN || j->ph == EULER)
		{
			get(0);
			j->r.res64 = (mpz_size(z) != 0) ? (uint64_t)mpz_getlimbn(z, 0) : 0;
			chunk_sum(j->res, j->E, j->B);
			ck(ab_set1(v));
			j->ph = GL_HI;
			j->i = (long)mpz_sizeinbase(j->res, 2) - 1;
			if (j->i >= j->B) { mpz_clear(z); return; }
		}
		if (j->ph == GL_HI)
		{
			ck(ab_mul(v, 0, 1));
			j->ph = GL_LO;
			j->i = j->B - 1;
			mpz_clear(z);
			return;
		}
		// GL_LO finished: a^res d(t)^(2^B) ?= d(t+1)
		mpz_t z2; mpz_init(z2);
		get(0);
		mpz_set(z2, z);
		get(2);
		const bool ok = mpz_cmp(z, z2) == 0;
		mpz_clears(z, z2, nullptr);
		ab_batch_release(c.b, slot);
		c.slots[slot] = nullptr;
		char msg[256];
		if (!ok) std::snprintf(msg, sizeof(msg), "Validation failed!");
		else if (j->r.is_prp) std::snprintf(msg, sizeof(msg), "N is a %s probable prime, a = %d.", j->euler ? "Euler" : "Fermat", j->a);
		else std::snprintf(msg, sizeof(msg), "N is composite, res64 = %s, a = %d.", hex64(j->r.res64).c_str(), j->a);
		finish(j, ok ? 0 : 1, msg);
	}

	// a test whose checks keep failing (a persistent fault) ends as failed
	void fail_repeated(Class & c, int slot, Job * j)
	{
		ab_batch_release(c.b, slot);
		c.slots[slot] = nullptr;
		finish(j, 1, "Validation failed repeatedly (Gerbicz-Li check).");
	}

	// queues one chunk of the class (asynchronous); returns false when idle
	bool launch_class(Class & c)
	{
		const int cap = c.cap, S = o.chunk;
		bool any = false;
		std::fill(c.mult.begin(), c.mult.end(), 0u);
		std::fill(c.snap.begin(), c.snap.end(), (uint8_t)0);
		std::vector<int> & count = c.count;
		count.assign(cap, 0);
		for (int s = 0; s < cap; ++s)
		{
			Job * j = c.slots[s];
			if (j == nullptr) continue;
			long n = std::min<long>(S, j->remaining());
			if (j->ph == MAIN && o.gl_check_blocks > 0)
			{
				// stop the chunk at the boundary where the next check is due
				const long next_b = (j->i / j->B) * j->B - (long)(o.gl_check_blocks - 1 - j->blocks) * j->B;
				if (next_b > 0 && next_b <= j->i) n = std::min<long>(n, j->i - next_b + 1);
			}
			count[s] = (int)n;
			for (long t = 0; t < n; ++t)
			{
				const long bit = j->i - t;
				c.mult[(size_t)t * cap + s] = j->mult_at(bit);
				if (j->ph == MAIN && bit % j->B == 0 && bit / j->B != 0) c.snap[(size_t)t * cap + s] = 1;
			}
			if (n > 0) any = true;
		}
		if (!any) return false;
		c.last_used = tick;
		ck(ab_batch_steps(c.b, S, c.mult.data(), c.snap.data()));
		return true;
	}

	// after the chunk: Gerbicz-Li products and the host steps between phases
	void settle_class(Class & c)
	{
		const int cap = c.cap;
		std::vector<int> & count = c.count;
		for (int s = 0; s < cap; ++s)
		{
			Job * j = c.slots[s];
			if (j == nullptr || count[s] == 0) continue;
			bool snapped = false;
			for (int t = 0; t < count[s]; ++t) snapped |= c.snap[(size_t)t * cap + s] != 0;
			const bool was_main = (j->ph == MAIN);
			const long last = j->i - count[s] + 1;             // the last bit this chunk processed
			bool check = false;
			if (snapped && o.gl_check_blocks > 0 && ++j->blocks >= o.gl_check_blocks && last % j->B == 0 && last > 0)
			{
				// d before this block's factor, for the check (a chunk holds at most
				// one boundary of a check: it stops there)
				ck(ab_copy(ab_batch_slot(c.b, s), 2, 1));
				check = true;
			}
			if (snapped) ck(ab_batch_gl_mul(c.b, s));
			j->i -= count[s];
			j->r.squarings += count[s];
			squarings += (uint64_t)count[s];
			if (was_main && !j->injected && o.inject_bit >= 0 && j->tag == o.inject_tag && last <= o.inject_bit)
			{
				// host-side fault: one word of Reg0 changes between two launches
				ck(ab_inject_word(ab_batch_slot(c.b, s), 0, o.inject_word, -1));
				j->injected = true;
			}
			if (check && j->remaining() > 0)
			{
				if (j->fails_in_row >= 8) { fail_repeated(c, s, j); continue; }
				j->chk_bit = last;
				start_check(ab_batch_slot(c.b, s), j);
				continue;
			}
			if (j->remaining() <= 0) next_phase(c, s, j);
		}
	}
};

extern "C" {

void ab_runner_options_default(ab_runner_options * o)
{
	std::memset(o, 0, sizeof(*o));
	o->hbm_budget_bytes = (size_t)32 << 30;
	o->max_slots_per_class = 256;
	o->chunk = 64;
	o->autotune = 1;
	o->gl_check_blocks = 0;
	o->inject_bit = -1;
}

int ab_runner_create(const ab_runner_options * o, ab_runner ** out)
{
	if (out == nullptr) return AB_E_ARG;
	ab_runner * r = new ab_runner();
	if (o) r->o = *o; else ab_runner_options_default(&r->o);
	if (r->o.chunk < 1 || r->o.max_slots_per_class < 1) { delete r; return AB_E_ARG; }
	*out = r;
	return AB_OK;
}

void ab_runner_destroy(ab_runner * r) { delete r; }

int ab_runner_submit(ab_runner * r, const uint64_t * Nl, size_t nlimbs, int euler, int32_t base, uint64_t tag)
{
	if (r == nullptr || Nl == nullptr || nlimbs == 0) return AB_E_ARG;
	Job * j = new Job();
	j->tag = tag;
	j->limbs.assign(Nl, Nl + nlimbs);
	mpz_import(j->N, nlimbs, -1, 8, 0, 0, Nl);
	j->euler = euler;
	j->a = (base != 0 && !euler) ? base : 2;
	j->r.base = j->a;
	r->queue.push_back(j);
	return AB_OK;
}

int ab_runner_advance(ab_runner * r, int * active, int * queued)
{
	if (r == nullptr) return AB_E_ARG;
	try
	{
		++r->tick;
		r->admit();
		std::vector<Class *> ran;
		for (auto & c : r->classes) if (r->launch_class(*c)) ran.push_back(c.get());
		for (Class * c : ran) r->settle_class(*c);
	}
	catch (const std::exception & e)
	{
		std::fprintf(stderr, "ab_runner_advance: %s\n", e.what());
		return AB_E_CUDA;
	}
	int a = 0;
	for (auto & c : r->classes) for (Job * j : c->slots) a += (j != nullptr);
	if (active) *active = a;
	if (queued) *queued = (int)r->queue.size();
	return AB_OK;
}

int ab_runner_synchronize(ab_runner * r)
{
	if (r == nullptr) return AB_E_ARG;
	for (auto & c : r->classes)
	{
		const int rc = ab_batch_synchronize(c->b);
		if (rc != AB_OK) return rc;
	}
	return AB_OK;
}

int ab_runner_poll(ab_runner * r, uint64_t * tag, ab_prp_result * out)
{
	if (r == nullptr || r->done.empty()) return 0;
	Job * j = r->done.front(); r->done.pop_front();
	if (tag) *tag = j->tag;
	if (out) *out = j->r;
	delete j;
	return 1;
}

int ab_runner_stats(const ab_runner * r, uint64_t * squarings, uint64_t * launches, int * batches)
{
	if (r == nullptr) return AB_E_ARG;
	uint64_t l = 0;
	for (auto & c : r->classes) { uint64_t x = 0; ab_batch_launch_count(c->b, &x); l += x; }
	if (squarings) *squarings = r->squarings;
	if (launches) *launches = l;
	if (batches) *batches = (int)r->classes.size();
	return AB_OK;
}

}
