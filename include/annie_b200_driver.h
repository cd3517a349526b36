/*
 * annie_b200 PRP test driver: the reference's annie::check
 * (src/annie.h:217-430) over the B200 transform, plus periodic Gerbicz-Li
 * verification with rollback to the last verified state and host-side fault
 * injection.  Host C++ (annie_b200/host/driver.cpp); numbers as LP64 limbs.
 */
#ifndef ANNIE_B200_DRIVER_H
#define ANNIE_B200_DRIVER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
	int euler;                 /* 1: Euler test, base = smallest non-square a with (a/N) = -1 (annie.h:249-253) */
	int32_t base;              /* Fermat base; 0 = the reference default 2 (annie.h:249, 254) */
	int device;
	int gl_check_blocks;       /* verify the Gerbicz-Li product every this many blocks of B squarings; 0 = final check only */
	int64_t inject_iteration;  /* flip one word of Reg0 right after this loop index (bit of the exponent); -1 = none */
	uint32_t inject_word;      /* index (mod 3 n) of the word of Reg0 to change (ab_inject_word) */
	const char * checkpoint_path;  /* NULL: no checkpoint files; else saved every checkpoint_seconds and on abort (annie.h:162-190) */
	double checkpoint_seconds;
	int verbose;
} ab_prp_options;

typedef struct
{
	int status;                /* 0 Success, 1 Failed (final Gerbicz-Li mismatch), 2 Aborted, -1 error */
	int decided_early;         /* 1: <= 15 digits, even, or a factor of R divides N (no exponentiation) */
	int is_prp;
	uint64_t res64;            /* low 64 bits of a^E' mod N (annie.h:364-366), E' = N - 1 */
	int32_t base;
	int K, pck, ln, lbase;
	int gl_block;              /* B (annie.h:97-101, 297) */
	int64_t squarings;         /* square_mul calls, including re-done and verification work */
	int gl_checks, gl_failures, rollbacks, resumed;
	double seconds;
	char message[256];         /* result line as the reference prints it */
} ab_prp_result;

void ab_prp_options_default(ab_prp_options * opt);

/* Full probable-prime test of N.  Returns status (also in out->status). */
int ab_prp_check(const uint64_t * N, size_t nlimbs, const ab_prp_options * opt, ab_prp_result * out);

/* Ask running tests to stop at the next iteration: they save a checkpoint
   (if configured) and return Aborted (the reference's quit(), annie.h:65-69). */
void ab_prp_quit(void);
void ab_prp_reset_quit(void);

/* One row of the benchmark table of the reference's -h mode (annie::bench,
   src/annie.h:432-556): N = 3 2^e + 1, base 3. */
typedef struct
{
	uint64_t e;
	int64_t digits;            /* decimal digits of N (mpz_sizeinbase(N, 10), as printed by the reference) */
	int K, pck, ln, lbase;
	int validated;             /* 1: the Gerbicz-Li check of the 6^50 exponentiation held; 0: test failed; -1: init failed */
	int64_t squarings;         /* timed square_mul calls */
	double ms_per_bit;         /* milliseconds per square_mul (one bit of the exponent) */
	double estimated_seconds;  /* ms_per_bit x bits of N: the time of a full test */
} ab_bench_row;

/* The reference's benchmark mode (annie::bench, src/annie.h:432-556) over the
   exponents e_list[0..count): for each, a Gerbicz-Li-validated exponentiation
   to 6^50 on a fresh transform, then `seconds` of squarings (the reference
   uses 10).  Stops after a row that does not validate, as the reference does;
   a row whose N shares a factor with the transform's R (validated = -1) is
   recorded and the table goes on.  Returns the rows written, or -1 on an
   error. */
int ab_bench_table(int device, const uint64_t * e_list, int count, double seconds, ab_bench_row * rows);

#ifdef __cplusplus
}
#endif

#endif
