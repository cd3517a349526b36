/*
 * annie_b200 batches and the continuous-batching runner -- no counterpart in
 * the reference, which tests one number at a time (src/annie.h:217-430).
 *
 * A batch is a size class (K, pck, ln) of `capacity` slots.  Each loaded slot
 * is a regular ab_transform (returned by ab_batch_slot: use it with ab_set1,
 * ab_copy, ab_mul, ab_get, ...; never ab_destroy it).  ab_batch_steps runs
 * `steps` squarings of every slot together from a captured CUDA graph.
 *
 * The runner queues PRP tests, admits them into batches as slots and HBM
 * budget free up, and runs each to its result (same verdict and RES64 as
 * ab_prp_check on the number alone).
 */
#ifndef ANNIE_B200_BATCH_H
#define ANNIE_B200_BATCH_H

#include <stddef.h>
#include <stdint.h>

#include "annie_b200.h"
#include "annie_b200_driver.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ab_batch ab_batch;

/* Device bytes one slot of the class holds. */
size_t ab_batch_slot_bytes(const ab_params * cls);
int ab_batch_create(int device, const ab_params * cls, int capacity, int max_steps, ab_batch ** out);
void ab_batch_destroy(ab_batch * b);
/* Sets up slot `slot` for N and base a (the digit size may differ between
   slots); N must fall in the class (K, pck, ln) by the factory rule. */
int ab_batch_load(ab_batch * b, int slot, const uint64_t * N, size_t nlimbs, int32_t a, int * init_failed);
/* ab_batch_load for `count` candidates at once: the host part of each load
   (parameters, N^-1 mod R, register words) runs on host threads, then the
   slots are set up on the device one after the other.  init_failed (nullable)
   receives one flag per candidate. */
int ab_batch_load_many(ab_batch * b, int count, const int * slots, const uint64_t * const * N, const size_t * nlimbs,
                       const int32_t * a, int * init_failed);
/* ab_batch_load in two halves, for schedulers that overlap set-up with
   squarings.  ab_batch_prepare is the host half (parameters, gcd(N, R),
   N^-1 mod R, register words: a GMP computation of about 0.5 s at 20 M bits);
   it makes no CUDA call and may run on any thread.  params (nullable)
   receives N's size class; init_failed (nullable) is 1 when gcd(N, R) != 1,
   and ab_prepared_factor then gives that gcd.  ab_batch_install is the device
   half; it takes ownership of p, also when it fails. */
typedef struct ab_prepared ab_prepared;
int ab_batch_prepare(const uint64_t * N, size_t nlimbs, int32_t a, ab_prepared ** out, ab_params * params, int * init_failed);
int ab_prepared_factor(const ab_prepared * p, uint64_t * out, size_t cap, size_t * count);
size_t ab_prepared_bytes(const ab_prepared * p);     /* host memory it holds */
void ab_prepared_destroy(ab_prepared * p);
int ab_batch_install(ab_batch * b, int slot, ab_prepared * p);
ab_transform * ab_batch_slot(ab_batch * b, int slot);
/* Slot dst becomes a copy of loaded slot src (same N and base, registers
   included) without the host set-up: for re-tests and throughput runs. */
int ab_batch_clone(ab_batch * b, int dst, int src);
int ab_batch_release(ab_batch * b, int slot);
/* mult[s * capacity + slot]: multiplier of squaring s for the slot (a or 1;
   0 = the slot sits this step out).  snap (nullable, same shape): after that
   squaring, keep Reg0 for the Gerbicz-Li product; ab_batch_gl_mul(slot) then
   does Reg1 *= kept value. */
int ab_batch_steps(ab_batch * b, int steps, const uint32_t * mult, const uint8_t * snap);
/* 2 when the batch's last chunk has completed, 1 when ab_batch_steps would
   queue its chunk without waiting (at most two chunks of a batch are in
   flight), 0 when it would wait, < 0 on error. */
int ab_batch_ready(const ab_batch * b);
int ab_batch_gl_mul(ab_batch * b, int slot);
/* Row levels per row pass (0 = default split); used by the autotuner. */
int ab_batch_set_geometry(ab_batch * b, int lb);
/* Autotuner: times `steps` batched squarings for every admissible row/column
   split of the class, with copies of slot `src` in the empty slots (released
   afterwards; the loaded slots are not touched), keeps the fastest split and
   remembers it for the process by (K, ln, capacity).  The reference picks its
   kernel split per length at compile time (transformGPU.h:403-470). */
int ab_batch_autotune(ab_batch * b, int src, int steps, int * row_levels);
int ab_batch_synchronize(ab_batch * b);
int ab_batch_launch_count(const ab_batch * b, uint64_t * count);

/* Mixed-size groups: batches of different size classes (NTT lengths up to
   2^20) squared together.  Each pass of a chunk is one launch over the
   candidates of every class of the group, which reads its per-class jobs
   from a device table; the slots' results are those of ab_batch_steps on
   each batch.  While in a group, a batch is stepped through the group only
   (its slots stay usable with every ab_transform call, and
   ab_batch_set_geometry makes the group re-record); destroy the group before
   its batches. */
typedef struct ab_mixed ab_mixed;
int ab_mixed_create(ab_batch * const * batches, int count, int max_steps, ab_mixed ** out);
void ab_mixed_destroy(ab_mixed * m);
/* mult[i], snap[i] (snap and snap[i] nullable): as ab_batch_steps for batch i. */
int ab_mixed_steps(ab_mixed * m, int steps, const uint32_t * const * mult, const uint8_t * const * snap);
/* As ab_batch_ready. */
int ab_mixed_ready(const ab_mixed * m);
int ab_mixed_synchronize(ab_mixed * m);
int ab_mixed_launch_count(const ab_mixed * m, uint64_t * count);

typedef struct ab_runner ab_runner;

typedef struct
{
	int device;
	size_t hbm_budget_bytes;   /* device memory the runner may give to batches */
	int max_slots_per_class;
	int chunk;                 /* squarings per graph launch */
	int autotune;              /* 1: tune the split of each new size class (ab_batch_autotune) */
	int gl_check_blocks;       /* verify each test's Gerbicz-Li product every this many blocks of B
	                              squarings and roll back to the last verified state on a mismatch
	                              (as ab_prp_check); 0 = only the final check of the reference */
	uint64_t inject_tag;       /* fault injection for tests: the test with this tag gets one word of
	                              Reg0 changed (ab_inject_word) once its loop passes bit inject_bit */
	int64_t inject_bit;        /* -1 = no injection */
	uint32_t inject_word;
	int latency_ln;            /* > 0: size classes with ln <= latency_ln (short squarings, latency-bound
	                              launches) and the larger ones take turns on the GPU in epochs of
	                              epoch_us microseconds, the larger ones with one chunk in flight, so
	                              that the short launches do not queue behind large grids; 0 = all
	                              classes run together */
	int epoch_us;
} ab_runner_options;

void ab_runner_options_default(ab_runner_options * o);
int ab_runner_create(const ab_runner_options * o, ab_runner ** out);
void ab_runner_destroy(ab_runner * r);
/* Queues a PRP test (Fermat base `base`, 0 = 2; or Euler). */
int ab_runner_submit(ab_runner * r, const uint64_t * N, size_t nlimbs, int euler, int32_t base, uint64_t tag);
/* Admits tests whose set-up is done into free slots, then queues one chunk of
   squarings for every batch that can take one without waiting (each batch
   keeps up to two in flight) and the host steps of the tests that reached the
   end of a phase.  Set-up (the Euler base, gcd(N, R), N^-1 mod R) runs on host
   threads of the runner, ahead of the free slots; when no test is on the GPU,
   the call waits for the set-ups in progress.  Returns within about 2 ms
   otherwise.  active: tests in slots; queued: tests submitted and not yet in a
   slot.  A test whose set-up fails (e.g. N too large) finishes with status -1
   and the error in its message. */
int ab_runner_advance(ab_runner * r, int * active, int * queued);
/* Waits for the work queued by ab_runner_advance on every batch. */
int ab_runner_synchronize(ab_runner * r);
/* Pops one finished test; returns 1 if one was available, 0 otherwise. */
int ab_runner_poll(ab_runner * r, uint64_t * tag, ab_prp_result * out);
/* Squarings executed for tests since creation (all slots). */
int ab_runner_stats(const ab_runner * r, uint64_t * squarings, uint64_t * launches, int * batches);

/* Per size class (batch) of the runner, for monitoring. */
typedef struct
{
	ab_params cls;             /* K, pck, ln (lbase 0) */
	int slots;                 /* capacity of the class's batch */
	int active;                /* tests in its slots */
	uint64_t squarings;        /* squarings run for its tests */
	uint64_t chunks;           /* chunks (graph launches) queued */
} ab_runner_class;
/* Fills up to cap entries; count receives the number of classes. */
int ab_runner_classes(const ab_runner * r, ab_runner_class * out, int cap, int * count);
/* Host seconds spent inside ab_runner_advance since creation: out[0]
   admission (installing set-ups, autotuning included), out[1] autotuning,
   out[2] host steps between phases, out[3] sleeping while no batch could
   take a chunk. */
int ab_runner_host_seconds(const ab_runner * r, double * out);

#ifdef __cplusplus
}
#endif

#endif
