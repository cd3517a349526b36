/*
 * TEST INFRASTRUCTURE ONLY (oracle).  Not part of the product.
 *
 * Thin C API over the reference implementation's OWN CPU code, compiled
 * unmodified from the reference sources:
 *   src/transformCPU.h   (class transformCPU, the CPU twin of the GPU engine)
 *   src/transformGMP.h   (class transformGMP, MMGW with GMP integers)
 *   src/annie.h          (class annie: the PRP test driver, built with CPU_TRANSFORM)
 * The reference expects <gmp.h>; annie_b200/gmp/gmp.h declares that API and
 * the system libgmp.so.10 provides it.  The Makefile in this folder builds
 * this file into oracle/_ref/libannie_ref.so.
 *
 * Nothing here reimplements reference logic: every call forwards to the
 * reference classes through the abstract `transform` interface
 * (src/transform.h:18-45).
 */
#include <cstdint>
#include <cstring>
#include <string>
#include <sstream>
#include <fstream>
#include <iostream>
#include <array>
#include <vector>
#include <memory>
#include <stdexcept>
#include <cstdio>
#include <unistd.h>
#include <sys/stat.h>

#include <gmp.h>

#define CPU_TRANSFORM true
#include "annie.h"

namespace
{
void mpz_from_limbs(mpz_t & z, const uint64_t * limbs, size_t n)
{
	mpz_import(z, n, -1, sizeof(uint64_t), 0, 0, limbs);
}

size_t mpz_to_limbs(const mpz_t & z, uint64_t * out, size_t cap)
{
	const size_t n = mpz_size(z);
	if (n > cap) return size_t(-1);
	for (size_t i = 0; i < n; ++i) out[i] = mpz_getlimbn(z, mp_size_t(i));
	return n;
}
}

extern "C" {

/* kind: 0 = transformCPU (K=5 NTT, src/transformCPU.h), 1 = transformGMP. */
void * ref_create(const uint64_t * n_limbs, size_t n_count, int32_t a, int kind)
{
	mpz_t N; mpz_init(N); mpz_from_limbs(N, n_limbs, n_count);
	transform * t = nullptr;
	try
	{
		if (kind == 0) t = new transformCPU(N, a);
		else t = new transformGMP(N, a);
	}
	catch (...) { t = nullptr; }
	mpz_clear(N);
	return t;
}

void ref_destroy(void * h) { delete static_cast<transform *>(h); }
int ref_init_failed(void * h) { return static_cast<transform *>(h)->init_failed() ? 1 : 0; }
void ref_set1(void * h) { static_cast<transform *>(h)->set1(); }
void ref_copy(void * h, size_t dst, size_t src) { static_cast<transform *>(h)->copy(dst, src); }
void ref_square_mul(void * h, int32_t a) { static_cast<transform *>(h)->square_mul(a); }
void ref_mul(void * h, size_t dst, size_t src) { static_cast<transform *>(h)->mul(dst, src); }

/* Runs `count` square_mul calls with the multipliers in `as` (one per call). */
void ref_square_mul_seq(void * h, const int32_t * as, size_t count)
{
	transform * t = static_cast<transform *>(h);
	for (size_t i = 0; i < count; ++i) t->square_mul(as[i]);
}

/* z = r_src (canonical, mod N); returns the limb count or -1 if cap is too small. */
long ref_get(void * h, size_t src, uint64_t * out, size_t cap)
{
	mpz_t z; mpz_init(z);
	static_cast<transform *>(h)->get(z, src);
	const size_t n = mpz_to_limbs(z, out, cap);
	mpz_clear(z);
	return (n == size_t(-1)) ? -1 : long(n);
}

void ref_get_factor(void * h, uint64_t * out, size_t cap, size_t * count)
{
	mpz_t z; mpz_init(z);
	static_cast<transform *>(h)->get_factor(z);
	*count = mpz_to_limbs(z, out, cap);
	mpz_clear(z);
}

/* copies get_info_short() into buf (NUL-terminated, truncated to cap) */
void ref_info(void * h, char * buf, size_t cap)
{
	const std::string s = static_cast<transform *>(h)->get_info_short();
	std::snprintf(buf, cap, "%s", s.c_str());
}

/* Writes the checkpoint payload (Reg0, Reg1) through the reference's own
   save_checkpoint into `path` (format of src/transformCPU.h:1475-1491). */
int ref_save_checkpoint(void * h, const char * path)
{
	transform * t = static_cast<transform *>(h);
	try
	{
		file f(path, "wb", true);
		t->save_checkpoint(f);
	}
	catch (...) { return -1; }
	return 0;
}

int ref_read_checkpoint(void * h, const char * path)
{
	transform * t = static_cast<transform *>(h);
	file f(path);
	if (!f.exists()) return -1;
	return t->read_checkpoint(f) ? 0 : -2;
}

/* Checkpoint files through the reference's own file class (src/file.h), in the
   layout of annie::save_checkpoint / _read_checkpoint (src/annie.h:140-181):
   int version = 1, int i, double elapsed, the transform payload, CRC-32 seal.
   write: 0 or -1.  read: 0, or -1 (no file), -2 (bad header or seal). */
int ref_file_write_checkpoint(const char * path, int i, double elapsed, const uint8_t * payload, size_t size)
{
	file f(path, "wb", false);
	if (!f.exists()) return -1;
	const int version = 1;
	if (!f.write(reinterpret_cast<const char *>(&version), sizeof(version))) return -1;
	if (!f.write(reinterpret_cast<const char *>(&i), sizeof(i))) return -1;
	if (!f.write(reinterpret_cast<const char *>(&elapsed), sizeof(elapsed))) return -1;
	if (!f.write(reinterpret_cast<const char *>(payload), size)) return -1;
	f.write_crc32();
	return 0;
}

int ref_file_read_checkpoint(const char * path, int * i, double * elapsed, uint8_t * payload, size_t size)
{
	file f(path);
	if (!f.exists()) return -1;
	int version = 0;
	if (!f.read(reinterpret_cast<char *>(&version), sizeof(version)) || version != 1) return -2;
	if (!f.read(reinterpret_cast<char *>(i), sizeof(*i))) return -2;
	if (!f.read(reinterpret_cast<char *>(elapsed), sizeof(*elapsed))) return -2;
	if (!f.read(reinterpret_cast<char *>(payload), size)) return -2;
	return f.check_crc32() ? 0 : -2;
}

/* The reference's own parameter rule for transformCPU (src/transformCPU.h:1493-1515). */
void ref_cpu_get_n_base(int * ln, int * lbase, int pck, double log2_16aN, double log2_p_2a)
{
	transformCPU::get_n_base(*ln, *lbase, pck, log2_16aN, log2_p_2a);
}

/* Full PRP test through the reference driver annie::check (src/annie.h:217-430)
   built with CPU_TRANSFORM.  Runs in `workdir` (the driver writes annie.log and
   results.txt in the current directory).  Returns 0 Success, 1 Failed,
   2 Aborted, -1 on exception. */
int ref_check(const uint64_t * n_limbs, size_t n_count, int is_euler, int a_ref, const char * workdir)
{
	char cwd[4096];
	if (getcwd(cwd, sizeof(cwd)) == nullptr) return -1;
	if (chdir(workdir) != 0) return -1;
	int ret = -1;
	try
	{
		mpz_t N; mpz_init(N); mpz_from_limbs(N, n_limbs, n_count);
		annie a;
		const annie::EReturn r = a.check(N, "N", is_euler != 0, a_ref, 0, true);
		ret = (r == annie::EReturn::Success) ? 0 : (r == annie::EReturn::Failed) ? 1 : 2;
		mpz_clear(N);
	}
	catch (...) { ret = -1; }
	if (chdir(cwd) != 0) return -1;
	return ret;
}

}
