/*
 * annie_b200: B200-native modular-squaring engine behind a C ABI.
 *
 * Drop-in for the reference's GPU transform (galloty/annie):
 *   class transform            src/transform.h:18-45     (the register machine)
 *   create_transformGPU(...)   src/transformGPU.h:822-885 (factory + parameter rule)
 *   transformGPU<LN>           src/transformGPU.h:286-796 (the engine the C++ host drives)
 * A C++ class implementing `transform` on top of these calls is in
 * annie_b200/host/transformCUDA.h.
 *
 * Numbers cross the ABI as little-endian arrays of 64-bit limbs (the layout of
 * GMP's mpz limbs on LP64).  Registers 0, 1, 2 are the reference's Reg0..Reg2.
 * Every function returns AB_OK (0) or a negative status; ab_last_error()
 * describes the last failure of the calling thread.  A handle is not
 * re-entrant: one host thread at a time per handle (as the reference).
 */
#ifndef ANNIE_B200_H
#define ANNIE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AB_OK              0
#define AB_E_ARG          -1   /* bad argument (register index, size, null pointer) */
#define AB_E_UNSUPPORTED  -2   /* NTT length outside the supported range */
#define AB_E_CUDA         -3   /* CUDA runtime error */
#define AB_E_INIT_FAILED  -4   /* gcd(N, R) != 1: see ab_get_factor (transformGPU.h:655-661) */
#define AB_E_CHECKPOINT   -5   /* checkpoint payload does not match K or n (transformGPU.h:608-624) */
#define AB_E_CAPACITY     -6   /* output buffer too small */
#define AB_E_TIMEOUT      -7   /* a device wait ran past its iteration limit */

typedef struct ab_transform ab_transform;

/* Transform parameters: K primes, packing pck = digits per coefficient,
   NTT length 2^ln, digit size 2^lbase (transformGPU.h:644-645). */
typedef struct
{
	int K, pck, ln, lbase;
} ab_params;

/* Parameter rule of create_transformGPU (transformGPU.h:822-857), or the
   forced parameters; init_failed = gcd(N, base^(pck n) - 1) != 1.  Host only. */
int ab_probe(const uint64_t * N, size_t nlimbs, int32_t a, const ab_params * forced,
	ab_params * out, int * init_failed);

/* create_transformGPU(N, a, device) (transformGPU.h:822) + constructor
   (transformGPU.h:644-753).  `forced` may be NULL.  If gcd(N, R) != 1 the
   handle is still created, ab_init_failed() returns 1 and ab_get_factor()
   gives the gcd (transformGPU.h:655-661, annie.h:269-283). */
int ab_create(const uint64_t * N, size_t nlimbs, int32_t a, int device, const ab_params * forced,
	ab_transform ** out);
void ab_destroy(ab_transform * h);                                   /* ~transformGPU (transformGPU.h:755-764) */

int ab_init_failed(const ab_transform * h);                          /* transform::init_failed (transform.h:32) */
int ab_get_factor(const ab_transform * h, uint64_t * out, size_t cap, size_t * count); /* transform::get_factor (transform.h:33) */
int ab_info(const ab_transform * h, ab_params * out);                /* transform::get_info_short (transformGPU.h:784-789) */

int ab_set1(ab_transform * h);                                       /* transform::set1  (transform.h:26, transformGPU.h:571-574) */
int ab_copy(ab_transform * h, size_t dst, size_t src);               /* transform::copy  (transform.h:28, transformGPU.h:588-591) */
int ab_square_mul(ab_transform * h, int32_t a);                      /* transform::square_mul (transform.h:29, transformGPU.h:593-596); a >= 1 */
int ab_mul(ab_transform * h, size_t dst, size_t src);                /* transform::mul   (transform.h:30, transformGPU.h:598-601) */
/* transform::get (transform.h:27, transformGPU.h:576-586): r_src out of
   MMGW form, reduced mod N; `count` = limbs written. */
int ab_get(ab_transform * h, size_t src, uint64_t * out, size_t cap, size_t * count);

/* transform::save_checkpoint / read_checkpoint (transform.h:37-38,
   transformGPU.h:608-641): payload = u32 K, u32 n, then per prime k the words
   of Reg0 and Reg1 (2n u32).  Size = 8 + 8 K n bytes. */
size_t ab_checkpoint_size(const ab_transform * h);
int ab_save_checkpoint(ab_transform * h, void * buf, size_t cap, size_t * written);
int ab_read_checkpoint(ab_transform * h, const void * buf, size_t size);

/* Page-locked host buffers for checkpoint payloads (DMA without staging). */
void * ab_host_alloc(size_t bytes);
void ab_host_free(void * p);

/* Raw register words of the reference's normal form: K planes of n u32, the
   residues of each coefficient's value mod the reference's primes -- the
   engine's read_memory / write_memory (engine.h of the reference).  The
   engine itself keeps each coefficient's exact value (three 32-bit limbs) and
   converts on the device; ab_write_register returns AB_E_ARG when the words
   are not those of a normal-form register (a coefficient beyond 96 bits). */
int ab_read_register(ab_transform * h, size_t reg, uint32_t * out, size_t cap_words);
int ab_write_register(ab_transform * h, size_t reg, const uint32_t * in, size_t nwords);

/* Fault injection for the Gerbicz-Li tests (no counterpart in the reference):
   adds delta to one 32-bit word (index mod 3 n) of the engine's own copy of
   register reg, between two launches. */
int ab_inject_word(ab_transform * h, size_t reg, size_t index, int32_t delta);

/* Waits for all work queued on the handle's stream. */
int ab_synchronize(ab_transform * h);

/* Runs `count` square_mul steps whose multipliers are `a` where the bit of
   `bits` (LSB first, bit i for step i) is set and 1 elsewhere -- the inner
   loop of annie::check (annie.h:319-341) without the Gerbicz-Li product.
   Full runs of 64 steps replay a captured CUDA graph (one launch instead of
   384); the rest are launched one by one. */
int ab_square_mul_bits(ab_transform * h, const uint64_t * bits, size_t count, int32_t a);

/* Row/column split of the NTT: `row_levels` radix-2 levels in the row pass,
   the other ln-1-row_levels in the column pass (at most 6).  Register
   contents are kept.  The reference fixes its split per length at compile
   time (transformGPU.h:403-470, forward/backward kernel choice); here it is
   a run-time choice for the autotuner.  AB_E_ARG if the split is not
   available for the length. */
int ab_set_geometry(ab_transform * h, int row_levels);
int ab_get_geometry(const ab_transform * h, int * row_levels, int * col_levels);

/* Schedule of a squaring: on != 0 (default) runs the Q-domain chain on a
   second stream beside the R-domain chain; on = 0 runs every launch on the
   handle's stream.  The registers do not depend on it (determinism tests). */
int ab_set_overlap(ab_transform * h, int on);

/* Device time of the work queued since the last call, in milliseconds
   (CUDA events on the handle's stream). */
int ab_timer_start(ab_transform * h);
int ab_timer_stop(ab_transform * h, float * ms);

const char * ab_last_error(void);

/* Number of kernels this handle has launched (all entry points). */
int ab_launch_count(const ab_transform * h, uint64_t * count);

/* Runs one square_mul(a) with a CUDA event before every kernel launch and
   returns each launch's device time (ms, launch order) in ms[0..*count).
   The launches are those of the overlapped schedule (one per domain: row
   and column pass of Q, of R, then the reduction), serialised on one
   stream so that each is timed alone. */
int ab_profile_square(ab_transform * h, int32_t a, float * ms, int cap, int * count);

/* Overwrites a device buffer of `bytes` (allocated on first use) on the
   handle's stream, evicting the transform's data from L2 (benchmarking). */
int ab_flush_l2(ab_transform * h, size_t bytes);

/* Allocation-free square_mul -- no counterpart in the reference.
 *
 * For callers that cannot allocate device memory once they are running: code
 * inside a stream capture (cudaMalloc is not capturable), a host that hands
 * all device memory to its own allocator or pool at start-up, or a service
 * with a fixed memory budget.  Such a caller creates the handle (which
 * allocates) during start-up, and afterwards squares registers it owns:
 * reg_device = a caller-owned device array of K*n words, a normal-form
 * register in the reference's layout (as ab_read_register gives it); it is
 * replaced by a * reg^2 in MMGW form, exactly as ab_square_mul does for Reg0.
 * The work buffers come from a static device array of 5 x 2^19 words
 * (10 MiB) that every GPU loading this library holds until exit, so the NTT
 * length must not exceed 2^16 (else AB_E_CAPACITY).  No
 * cudaMalloc, cudaFree or allocating library call is made: the array's device
 * address is looked up (cudaGetSymbolAddress, with the device current) when
 * the handle is created, so a call only queues kernels.  a must be >= 1
 * (else AB_E_ARG).  Work is queued on the handle's stream (ab_synchronize
 * waits for it).  All
 * calls share the one array: calls whose work overlaps on the GPU (other
 * handles' streams, other host threads) race and give wrong results. */
int ab_square_mul_noalloc(ab_transform * h, uint32_t * reg_device, int32_t a);

/* Diagnostics (kernel-level parity tests): run one stage on host data; inputs
   and the product's output are normal-form registers in the reference's
   layout (K planes).  They use the handle's work buffers (registers kept).
   ab_diag_forward:  full forward NTT of a register (domain 0 = R, 1 = Q) over
                     the engine's own transform primes: (K+1) planes of n
                     lazily reduced residues.
   ab_diag_product:  forward NTT, pointwise square (y == NULL) or product with
                     register y, inverse NTT, carry (a, nega for domain Q,
                     optional subtraction, lower_mode 0 none / 1 mod R + 2 / 2 mod Q). */
int ab_diag_forward(ab_transform * h, int domain, const uint32_t * in, uint32_t * out);
int ab_diag_product(ab_transform * h, int domain, const uint32_t * in, const uint32_t * y,
	uint32_t a, const uint32_t * sub, int lower_mode, uint32_t * out);

#ifdef __cplusplus
}
#endif

#endif
