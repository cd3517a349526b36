// Launch interface of the NTT passes (host side).
//
// Transform layout: one register = K planes of n = 2^ln residues (plane k at
// offset k*n).  The length-n negacyclic/cyclic NTT of the reference
// (ocl/kernel.cl: LN-1 radix-2 levels, then a pointwise product of degree-1
// polynomials) is split 2-D: coefficient i = row*R + col, H rows, R columns.
//   * column pass (k_colpass): the first LA = log2(H) levels (strides >= R),
//     fused with the inverse of those levels, the carry of the previous product
//     and the first levels of the next product;
//   * row pass (k_rowpass): the last LB levels (strides < R), the pointwise
//     square / multiply, and the inverse of those LB levels, one CTA per row.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "arith.cuh"

namespace ab
{

enum RowMode { ROW_FWD_ONLY = 0, ROW_SQUARE = 1, ROW_MUL = 2 };

// Batches: blockIdx.z selects a candidate; its buffers are at +z*stride
// words (twiddles are shared).  `active` (nullable) holds one word per
// candidate, 0 = skip it.
struct RowJob
{
	u32 * x;          // K x n buffer, rows transformed in place
	const u32 * xp;   // ROW_MUL: pre-transformed operand (same layout)
	const u32 * w;    // twiddles of the domain: per prime n words, w (n/2) || wi (n/2)
	int mode;
	size_t stride;
	const u32 * active;
};
struct RowJobs { RowJob j[2]; };

enum LowerMode { LOWER_NONE = 0, LOWER_R_ADD2 = 1, LOWER_Q = 2 };

struct ColJob
{
	const u32 * in;      // source buffer
	int transformed;     // 1: source awaits the inverse column levels + carry; 0: normal-form residues
	const u32 * w_in;    // twiddles of the source domain (transformed source)
	u32 a;               // carry: multiply by a
	int nega;            // carry: wrap-around negated (mod x^n + 1)
	const u32 * sub;     // carry: subtract this normal-form register (nullable)
	int sub_big;         // 1: `sub` holds exact coefficient values (K two's-complement limbs per coefficient, as out_big writes)
	int lower;           // LowerMode applied after the carry
	u32 * out_norm;      // normal-form result (nullable)
	int out_big;         // 1: out_norm receives each coefficient's exact value (K limbs, plane k = limb k)
	                     // instead of its residues -- for T_Q, which only the subtracting carry reads
	u32 * out_fwd[2];    // first LA forward levels of the result, per domain (nullable)
	const u32 * w_out[2];
	size_t stride;       // words between candidates (batches)
	const u32 * mult;    // per candidate: the carry multiplier a, 0 = inactive (nullable: use `a`)
	const CandConst * cand;  // per-candidate digit constants (nullable: those of TConst)
	u32 * out_snap;      // per candidate: also store the normal form here when snap_flag[z] != 0
	const u32 * snap_flag;
};
struct ColJobs { ColJob j[2]; };

struct Geometry
{
	int ln, LA, LB;
	u32 H, R;
	int C;               // columns per column-pass CTA
};

// Chooses the 2-D split for a transform of length 2^ln (6 <= ln <= 21).
bool make_geometry(int ln, int lb_override, Geometry & g);

// Column-pass scratch in shared memory, bytes.
size_t colpass_smem(const Geometry & g, int K);

cudaError_t launch_rowpass(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s, int ncand = 1);
cudaError_t launch_colpass(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s, int ncand = 1);

} // namespace ab
