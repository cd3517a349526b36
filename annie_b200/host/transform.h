// The register-machine interface the PRP driver programs against -- the same
// abstract class as the reference's src/transform.h:18-45 (names and meaning
// kept so that a driver written for it runs unchanged on this engine).
#pragma once

#include <cstdint>
#include <string>

#include "gmp.h"
#include "ckfile.h"

class transform
{
public:
	static const size_t Reg0 = 0, Reg1 = 1, Reg2 = 2;

	virtual void set1() = 0;                                      // r_0 = 1 (MMGW form)
	virtual void get(mpz_t & z, const size_t src) = 0;            // z = r_src mod N
	virtual void copy(const size_t dst, const size_t src) = 0;    // r_dst = r_src
	virtual void square_mul(const int32_t a) = 0;                 // r_0 = a * r_0^2
	virtual void mul(const size_t dst, const size_t src) = 0;     // r_dst *= r_src
	virtual bool init_failed() const = 0;
	virtual void get_factor(mpz_t & z) const = 0;

	virtual bool has_checkpoint() const = 0;
	virtual bool read_checkpoint(ckfile & cfile) = 0;              // r_0 and r_1
	virtual void save_checkpoint(ckfile & cfile) = 0;              // r_0 and r_1

	transform() {}
	virtual ~transform() {}

	virtual std::string get_type() const = 0;
	virtual std::string get_data_size() const = 0;
	virtual std::string get_cache_size() const = 0;
	virtual std::string get_info_short() const = 0;
	virtual std::string get_info() const = 0;
};
