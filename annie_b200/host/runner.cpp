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
//
// Admission is a pipeline: set-up threads classify each submitted test and
// do the host half of its slot's set-up (gcd(N, R), N^-1 mod R: about 0.5 s
// of GMP at 20 M bits) while the GPU squares the admitted ones; advance()
// installs finished set-ups into free slots.  Each size class keeps up to two
// chunks in flight on its own stream and is relaunched as soon as it can be,
// so small classes are not held to the pace of large ones.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
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

	// admission, written by a set-up thread and read by the runner once the
	// job is handed back: decided without a transform (early, with its
	// message), the host half of the slot's set-up and N's size class, or
	// the error that set-up met
	bool early = false;
	std::string early_msg;
	ab_prepared * prep = nullptr;
	ab_params p{};
	int gcd_failed = 0;
	int prep_rc = AB_OK;
	std::string prep_err;

	Job() { mpz_inits(N, E, res, chk, nullptr); }
	~Job() { ab_prepared_destroy(prep); mpz_clears(N, E, res, chk, nullptr); }

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
	uint64_t squarings = 0, chunks = 0;
};

using clk = std::chrono::steady_clock;
double secs(clk::duration d) { return std::chrono::duration<double>(d).count(); }

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
	std::deque<Job *> queue;           // submitted, not yet handed to set-up
	std::deque<Job *> done;
	std::vector<std::unique_ptr<Class>> classes;
	size_t used = 0;
	uint64_t squarings = 0;
	uint64_t tick = 0;                 // advance() calls

	// set-up threads and their queues
	std::vector<std::thread> workers;
	std::mutex mu;
	std::condition_variable cv_work, cv_ready;
	std::deque<Job *> todo, ready;     // guarded by mu
	int working = 0;                   // guarded by mu
	bool stopping = false;             // guarded by mu
	std::deque<Job *> prepared;        // set up, waiting for a slot
	size_t outstanding = 0;            // handed to set-up, not yet in a slot or decided
	size_t prepared_bytes = 0;         // host memory held by `prepared`
	double host_s[4] = {};             // advance(): admission, autotune, host steps, waiting

	// latency epochs (latency_ln > 0): whose turn it is, since when
	bool small_turn = true;
	clk::time_point epoch_t0{};

	bool is_small(const Class & c) const { return c.cls.ln <= o.latency_ln; }

	static bool has_tests(const Class & c)
	{
		return std::any_of(c.slots.begin(), c.slots.end(), [](Job * j) { return j != nullptr; });
	}

	// the turn passes to the other group when its epoch is over or it has no
	// tests left
	void pick_turn()
	{
		bool has[2] = {false, false};
		for (auto & c : classes) if (has_tests(*c)) has[is_small(*c) ? 1 : 0] = true;
		const auto now = clk::now();
		const bool other = has[small_turn ? 0 : 1], mine = has[small_turn ? 1 : 0];
		if (other && (!mine || now - epoch_t0 > std::chrono::microseconds(o.epoch_us)))
		{
			small_turn = !small_turn;
			epoch_t0 = now;
		}
	}

	// set-up runs at most this far ahead of the free slots
	static constexpr size_t max_ahead = 1024;
	static constexpr size_t max_ahead_bytes = size_t(1) << 30;

	~ab_runner()
	{
		{
			std::lock_guard<std::mutex> lk(mu);
			stopping = true;
		}
		cv_work.notify_all();
		for (auto & t : workers) t.join();
		for (auto & c : classes)
		{
			for (Job * j : c->slots) delete j;
			ab_batch_destroy(c->b);
		}
		for (auto * q : {&queue, &done, &todo, &ready, &prepared})
			for (Job * j : *q) delete j;
	}

	void finish(Job * j, int status, const char * msg)
	{
		j->r.status = status;
		std::snprintf(j->r.message, sizeof(j->r.message), "%s", msg);
		j->ph = DONE;
		done.push_back(j);
	}

	// set-up thread: trivial cases, the Euler base, then the host half of the
	// slot's set-up (no CUDA call here)
	static void prepare_job(Job * j)
	{
		const mpz_srcptr n = j->N;
		if (mpz_sizeinbase(n, 2) <= 50 && mpz_cmp_ui(n, 999999999999999ul) <= 0)
		{
			const int pp = mpz_probab_prime_p(n, 20);
			j->r.decided_early = 1;
			j->r.is_prp = pp != 0;
			j->early = true;
			j->early_msg = (pp != 0) ? "N is a probable prime." : "N is composite.";
			return;
		}
		if (mpz_even_p(n)) { j->r.decided_early = 1; j->early = true; j->early_msg = "N is even."; return; }
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
		j->prep_rc = ab_batch_prepare(j->limbs.data(), j->limbs.size(), j->a, &j->prep, &j->p, &j->gcd_failed);
		if (j->prep_rc != AB_OK) j->prep_err = ab_last_error();
	}

	void worker()
	{
		std::unique_lock<std::mutex> lk(mu);
		for (;;)
		{
			cv_work.wait(lk, [&] { return stopping || !todo.empty(); });
			if (stopping) return;
			Job * j = todo.front(); todo.pop_front();
			++working;
			lk.unlock();
			prepare_job(j);
			lk.lock();
			--working;
			ready.push_back(j);
			cv_ready.notify_all();
		}
	}

	// hands queued tests to the set-up threads, as far ahead as the bounds allow
	void feed()
	{
		std::vector<Job *> batch;
		while (!queue.empty() && outstanding < max_ahead && prepared_bytes < max_ahead_bytes)
		{
			batch.push_back(queue.front());
			queue.pop_front();
			++outstanding;
		}
		if (batch.empty()) return;
		if (workers.empty())
		{
			const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
			const unsigned nt = std::min(16u, std::max(1u, hw / 2));
			for (unsigned t = 0; t < nt; ++t) workers.emplace_back([this] { worker(); });
		}
		{
			std::lock_guard<std::mutex> lk(mu);
			for (Job * j : batch) todo.push_back(j);
		}
		cv_work.notify_all();
	}

	// takes the finished set-ups; with wait_all, first waits until the set-up
	// threads have none left (the GPU has nothing to run meanwhile)
	void collect(bool wait_all)
	{
		std::deque<Job *> got;
		{
			std::unique_lock<std::mutex> lk(mu);
			if (wait_all) cv_ready.wait(lk, [&] { return todo.empty() && working == 0; });
			got.swap(ready);
		}
		for (Job * j : got)
		{
			prepared.push_back(j);
			prepared_bytes += ab_prepared_bytes(j->prep);
		}
	}

	size_t live_slots() const
	{
		size_t a = 0;
		for (auto & c : classes) for (Job * j : c->slots) a += (j != nullptr);
		return a;
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

	// Admission: the set-up tests go into free slots of their size class (a
	// class is created within the HBM budget), in submission order; the
	// others wait for a slot
	void install()
	{
		std::deque<Job *> later;
		while (!prepared.empty())
		{
			Job * j = prepared.front(); prepared.pop_front();
			if (j->early || j->prep_rc != AB_OK || j->gcd_failed)
			{
				prepared_bytes -= ab_prepared_bytes(j->prep);
				--outstanding;
				if (j->early) { finish(j, 0, j->early_msg.c_str()); continue; }
				if (j->prep_rc != AB_OK)
				{
					const std::string m = "the test could not be set up: " + j->prep_err;
					finish(j, -1, m.c_str());
					continue;
				}
				std::vector<uint64_t> f(j->limbs.size() + 2);
				size_t fc = 0;
				ck(ab_prepared_factor(j->prep, f.data(), f.size(), &fc));
				mpz_t z; mpz_init(z); mpz_import(z, fc, -1, 8, 0, 0, f.data());
				char * str = mpz_get_str(nullptr, 10, z);
				char msg[256]; std::snprintf(msg, sizeof(msg), "%.200s divides N.", str);
				free(str); mpz_clear(z);
				j->r.decided_early = 1;
				finish(j, 0, msg);
				continue;
			}
			const ab_params & p = j->p;
			j->r.K = p.K; j->r.pck = p.pck; j->r.ln = p.ln; j->r.lbase = p.lbase;
			Class * c = class_for(p, true);
			if (c == nullptr) { later.push_back(j); continue; }
			const int slot = (int)(std::find(c->slots.begin(), c->slots.end(), nullptr) - c->slots.begin());
			prepared_bytes -= ab_prepared_bytes(j->prep);
			--outstanding;
			ab_prepared * pp = j->prep;
			j->prep = nullptr;
			if (ab_batch_install(c->b, slot, pp) != AB_OK)
			{
				// the test ends with the error; the ones still waiting stay queued
				const std::string m = std::string("the test could not be set up on the device: ") + ab_last_error();
				finish(j, -1, m.c_str());
				for (Job * w : prepared) later.push_back(w);
				prepared.swap(later);
				throw rt_error(m);
			}
			c->slots[slot] = j;
			ab_transform * v = ab_batch_slot(c->b, slot);
			ck(ab_set1(v));
			ck(ab_copy(v, 1, 0));
			if (!c->tuned)
			{
				int lb = 0;
				const auto t0 = clk::now();
				// 16 squarings per split are enough to rank the splits
				if (o.autotune) ck(ab_batch_autotune(c->b, slot, std::min(o.chunk, 16), &lb));
				host_s[1] += secs(clk::now() - t0);
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
		prepared.swap(later);
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
		++c.chunks;
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
			c.squarings += (uint64_t)count[s];
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
			if (j->remaining() <= 0)
			{
				const auto t0 = clk::now();
				next_phase(c, s, j);
				host_s[2] += secs(clk::now() - t0);
			}
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
	o->latency_ln = 0;
	o->epoch_us = 20000;
}

int ab_runner_create(const ab_runner_options * o, ab_runner ** out)
{
	if (out == nullptr) return AB_E_ARG;
	ab_runner * r = new ab_runner();
	if (o) r->o = *o; else ab_runner_options_default(&r->o);
	if (r->o.chunk < 1 || r->o.max_slots_per_class < 1 || r->o.latency_ln < 0 || (r->o.latency_ln > 0 && r->o.epoch_us < 1))
	{
		delete r;
		return AB_E_ARG;
	}
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
		r->feed();
		// with nothing on the GPU, wait for the set-ups in progress
		const auto ta = clk::now();
		r->collect(r->live_slots() == 0 && r->outstanding > r->prepared.size());
		r->install();
		r->feed();
		r->host_s[0] += secs(clk::now() - ta);
		// one chunk for every class that can take one without waiting; when
		// none can, poll for up to 2 ms
		// (with latency epochs, only the classes whose turn it is, the large
		// ones when their last chunk is done)
		const bool epochs = r->o.latency_ln > 0;
		const auto t0 = std::chrono::steady_clock::now();
		for (;;)
		{
			bool launched = false, busy = false;
			if (epochs) r->pick_turn();
			for (auto & c : r->classes)
			{
				if (!ab_runner::has_tests(*c)) continue;
				busy = true;
				if (epochs && r->is_small(*c) != r->small_turn) continue;
				const int rd = ab_batch_ready(c->b);
				if (rd < 0) throw rt_error(ab_last_error());
				if (rd == 0 || (epochs && !r->is_small(*c) && rd < 2)) continue;
				if (r->launch_class(*c)) { r->settle_class(*c); launched = true; }
			}
			if (launched || !busy) break;
			if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(2)) break;
			const auto tw = clk::now();
			std::this_thread::sleep_for(std::chrono::microseconds(20));
			r->host_s[3] += secs(clk::now() - tw);
		}
	}
	catch (const std::exception & e)
	{
		std::fprintf(stderr, "ab_runner_advance: %s\n", e.what());
		return AB_E_CUDA;
	}
	if (active) *active = (int)r->live_slots();
	if (queued) *queued = (int)(r->queue.size() + r->outstanding);
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

int ab_runner_classes(const ab_runner * r, ab_runner_class * out, int cap, int * count)
{
	if (r == nullptr || count == nullptr || (cap > 0 && out == nullptr)) return AB_E_ARG;
	int i = 0;
	for (auto & c : r->classes)
	{
		if (i < cap)
		{
			ab_runner_class & x = out[i];
			x.cls = c->cls;
			x.slots = c->cap;
			x.active = (int)std::count_if(c->slots.begin(), c->slots.end(), [](Job * j) { return j != nullptr; });
			x.squarings = c->squarings;
			x.chunks = c->chunks;
		}
		++i;
	}
	*count = i;
	return AB_OK;
}

int ab_runner_host_seconds(const ab_runner * r, double * out)
{
	if (r == nullptr || out == nullptr) return AB_E_ARG;
	for (int i = 0; i < 4; ++i) out[i] = r->host_s[i];
	return AB_OK;
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
