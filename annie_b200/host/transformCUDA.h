// transformCUDA: the `transform` register machine on a B200, over the C ABI
// of include/annie_b200.h.  It takes the place of the reference's
// transformGPU<LN> (src/transformGPU.h:286-796) and of its factory
// create_transformGPU (src/transformGPU.h:822-885): same parameter rule,
// same registers, same checkpoint payload, same error conditions (thrown as
// std::runtime_error, as the reference's OpenCL layer does).
#pragma once

#include <cstdint>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <vector>

#include "gmp.h"
#include "transform.h"
#include "../../include/annie_b200.h"

class transformCUDA : public transform
{
	ab_transform * _h = nullptr;
	ab_params _p{};
	mpz_t _N;
	size_t _nlimbs = 0;
	std::vector<uint64_t> _bits;

	static void check(int rc)
	{
		if (rc != AB_OK) throw std::runtime_error(std::string("annie_b200: ") + ab_last_error());
	}

public:
	transformCUDA(mpz_srcptr N, int32_t a, int device, const ab_params * forced = nullptr)
	{
		mpz_init_set(_N, N);
		_nlimbs = mpz_size(N);
		std::vector<uint64_t> limbs(_nlimbs);
		for (size_t i = 0; i < _nlimbs; ++i) limbs[i] = mpz_getlimbn(N, (mp_size_t)i);
		check(ab_create(limbs.data(), _nlimbs, a, device, forced, &_h));
		check(ab_info(_h, &_p));
	}

	~transformCUDA() override
	{
		ab_destroy(_h);
		mpz_clear(_N);
	}

	ab_transform * handle() const { return _h; }
	const ab_params & params() const { return _p; }

	void set1() override { check(ab_set1(_h)); }
	void copy(size_t dst, size_t src) override { check(ab_copy(_h, dst, src)); }
	void square_mul(int32_t a) override { check(ab_square_mul(_h, a)); }

	// `count` square_mul steps over the bits of e from bit `top` downwards:
	// step s multiplies by a when bit top - s of e is set (one call, runs of
	// steps replayed from a CUDA graph)
	void square_mul_bits(const mpz_t e, long top, long count, int32_t a)
	{
		if (count <= 0) return;
		_bits.assign((size_t)(count + 63) / 64, 0);
		for (long s = 0; s < count; ++s)
		{
			const long bit = top - s;
			if (bit >= 0 && mpz_tstbit(e, (mp_bitcnt_t)bit)) _bits[(size_t)s / 64] |= uint64_t(1) << (s % 64);
		}
		check(ab_square_mul_bits(_h, _bits.data(), (size_t)count, a));
	}
	void mul(size_t dst, size_t src) override { check(ab_mul(_h, dst, src)); }

	void get(mpz_t & z, size_t src) override
	{
		std::vector<uint64_t> out(_nlimbs + 2);
		size_t cnt = 0;
		check(ab_get(_h, src, out.data(), out.size(), &cnt));
		mpz_import(z, cnt, -1, 8, 0, 0, out.data());
	}

	bool init_failed() const override { return ab_init_failed(_h) != 0; }

	void get_factor(mpz_t & z) const override
	{
		std::vector<uint64_t> out(_nlimbs + 2);
		size_t cnt = 0;
		check(ab_get_factor(_h, out.data(), out.size(), &cnt));
		mpz_import(z, cnt, -1, 8, 0, 0, out.data());
	}

	bool has_checkpoint() const override { return true; }

	// payload of transformGPU.h:608-641: u32 K, u32 n, then per prime Reg0 || Reg1
	std::vector<uint8_t> payload()
	{
		std::vector<uint8_t> buf(ab_checkpoint_size(_h));
		size_t w = 0;
		check(ab_save_checkpoint(_h, buf.data(), buf.size(), &w));
		return buf;
	}

	bool load_payload(const std::vector<uint8_t> & buf)
	{
		const int rc = ab_read_checkpoint(_h, buf.data(), buf.size());
		if (rc == AB_E_CHECKPOINT) return false;
		check(rc);
		return true;
	}

	bool read_checkpoint(ckfile & f) override
	{
		uint32_t hdr[2];
		if (!f.read(hdr, sizeof(hdr))) return false;
		std::vector<uint8_t> buf(ab_checkpoint_size(_h));
		if (buf.size() < 8) return false;
		std::memcpy(buf.data(), hdr, 8);
		if (hdr[0] != (uint32_t)_p.K || hdr[1] != (uint32_t)(1u << _p.ln)) return false;
		if (!f.read(buf.data() + 8, buf.size() - 8)) return false;
		return load_payload(buf);
	}

	void save_checkpoint(ckfile & f) override
	{
		const std::vector<uint8_t> buf = payload();
		f.write(buf.data(), buf.size());
	}

	std::string get_type() const override { return "CUDA sm_100a"; }

	std::string get_data_size() const override
	{
		// 7 normal-form buffers (3 words per coefficient), 8 NTT-form buffers and
		// 3 twiddle tables (K + 1 words), the reference-word staging (K words)
		const size_t bytes = (size_t)(21 + 11 * (_p.K + 1) + _p.K) * ((size_t)1 << _p.ln) * 4;
		std::ostringstream ss; ss << "data size: ";
		if (bytes < (10u << 20)) ss << bytes / 1024 << " KB"; else ss << (bytes >> 20) << " MB";
		return ss.str();
	}

	std::string get_cache_size() const override { return "cache size: 0 KB"; }

	std::string get_info_short() const override
	{
		std::ostringstream ss;
		ss << _p.K + 1 << "-prime NTT of length " << (1u << _p.ln) << ", packed-base = 2^{" << _p.pck << "x" << _p.lbase << "}";
		return ss.str();
	}

	std::string get_info() const override
	{
		return "Montgomery-McLaughlin-Gallot-Woltman reduction, " + get_info_short() + "\n";
	}
};
