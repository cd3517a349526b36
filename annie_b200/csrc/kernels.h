// Launch interface of the NTT passes (host side).
//
// Layouts (all words u32):
// * NTT form: KP planes of n = 2^ln lazy residues mod the transform primes
//   (plane k at offset k*n).  The length-n cyclic (domain R, x^n - 1) or
//   negacyclic (domain Q, x^n + 1) transform is ln - 1 radix-2 levels that
//   split the register into n/2 polynomials of degree 1 (ocl/kernel.cl), split
//   2-D: coefficient i = row*R + col, H rows, R columns.
//     * column pass (k_colpass): the first LA = log2(H) levels (strides >= R),
//       fused with the inverse of those levels, the carry of the previous
//       product and the first levels of the next product;
//     * row pass (k_rowpass): the last LB levels (strides < R), the pointwise
//       square / multiply, and the inverse of those LB levels, one CTA per row.
// * Normal form: AB_NW = 3 planes of n words, the limbs (low first) of each
//   coefficient's exact value in two's complement.
// * Twiddles of one domain and prime, at the reference's bit-reversed
//   positions (level with s polynomials: index s + bitrev(j, s), s = n/4 .. 1):
//     - row tables: n/2 Shoup pairs (w, floor(w 2^32/p)), forward w; domain R
//       also has -w^-1.  Domain Q needs no inverse table: there
//       -w_j^-1 = w_{s-1-j}, the forward twiddle at the mirrored position.
//     - column tables: the first COLTW positions (the column levels), forward
//       and -w^-1, for both domains, as Shoup pairs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "arith.cuh"

namespace ab
{

enum RowMode { ROW_FWD_ONLY = 0, ROW_SQUARE = 1, ROW_MUL = 2 };

constexpr int COLTW = 128;   // column-table positions per prime (covers H <= 64 and its mirror)

// Batches: blockIdx.z selects a candidate; its buffers are at +z*stride
// words (twiddles are shared).  `active` (nullable) holds one word per
// candidate, 0 = skip it.
struct RowJob
{
	u32 * x;          // KP x n buffer, rows transformed in place
	const u32 * xp;   // ROW_MUL: full forward image of the other operand (same layout)
	const uint2 * w;  // row table of the domain: per prime n/2 Shoup pairs
	const uint2 * wi; // domain R: its -w^-1 row table; null = domain Q (mirrored w)
	int mode;
	size_t stride;    // words between candidates (x and xp)
	const u32 * active;
};
struct RowJobs { RowJob j[2]; };

enum LowerMode { LOWER_NONE = 0, LOWER_R_ADD2 = 1, LOWER_Q = 2 };

struct ColJob
{
	const u32 * in;      // source buffer
	int transformed;     // 1: NTT-form source awaiting the inverse column levels + carry; 0: normal form
	const uint2 * wi_in; // column table -w^-1 of the source domain (transformed source), COLTW pairs per prime
	u32 a;               // carry: multiply by a
	int nega;            // carry: wrap-around negated (mod x^n + 1)
	const u32 * sub;     // carry: subtract this normal-form register (nullable)
	int lower;           // LowerMode applied after the carry
	u32 * out_norm;      // normal-form result (nullable)
	u32 * out_fwd[2];    // first LA forward levels of the result, per domain (nullable)
	const uint2 * w_out[2];  // forward column tables of the output domains
	size_t stride_ntt;   // words between candidates of NTT-form buffers (in when transformed, out_fwd)
	size_t stride_norm;  // words between candidates of normal-form buffers (in when not, sub, out_norm, out_snap)
	const u32 * mult;    // per candidate: the carry multiplier a, 0 = inactive (nullable: use `a`)
	const CandConst * cand;  // per-candidate digit size (nullable: that of TConst)
	u32 * out_snap;      // per candidate: also store the normal form here when snap_flag[z] != 0
	const u32 * snap_flag;
};
struct ColJobs { ColJob j[2]; };

// Split of the ln - 1 levels: LA column levels, G mid levels, LB row levels.
// Coefficient i = (h 2^G + m) R + c with h < H = 2^LA rows for the column
// pass (whose rows are RC = R 2^G words), m < 2^G, and c < R = 2^(LB+1); the
// row pass sees HR = H 2^G rows of R words.  G > 0 only above 2^20.
struct Geometry
{
	int ln, LA, LB, G;
	u32 H, R, HR, RC;
	int C;               // columns per column-pass CTA
};

// Chooses the split for a transform of length 2^ln (6 <= ln <= 22);
// lb_override > 0 asks for that many row levels.
bool make_geometry(int ln, int lb_override, Geometry & g);

// The launch constants that describe a split.
inline void apply_geometry(TConst & c, const Geometry & g)
{
	c.R = g.RC; c.H = g.H; c.HR = g.HR; c.LA = g.LA; c.LB = g.LB; c.G = g.G;
}

// Column-pass scratch in shared memory, bytes.
size_t colpass_smem(const Geometry & g, int KP);

cudaError_t launch_rowpass(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s, int ncand = 1);
// The G mid levels of the row jobs' buffers, forward or inverse (G > 0).
cudaError_t launch_midpass(const Geometry & g, const TConst & c, const RowJobs & jobs, int njobs, cudaStream_t s, int ncand, bool inverse);
cudaError_t launch_colpass(const Geometry & g, const TConst & c, const ColJobs & jobs, int njobs, cudaStream_t s, int ncand = 1);

// Mixed-size passes: one launch runs the same pass for the candidates of
// several size classes (lengths up to 2^20, no mid levels).  CTAs
// [begin[i], begin[i+1]) belong to class i, nbx per job and candidate
// (candidate-major, then job); each class has its own constants (tcs[i]),
// jobs and row or column split.
constexpr int AB_FUSE_MAXC = 16;
constexpr unsigned AB_FUSED_ROW_THREADS = 256;
struct FusedRowPass
{
	int nclass;
	u32 begin[AB_FUSE_MAXC + 1];
	u32 nbx[AB_FUSE_MAXC];        // KP HR rows
	u32 njobs[AB_FUSE_MAXC];
	int log_r[AB_FUSE_MAXC];      // row length 2^log_r (LB + 1)
	RowJobs jobs[AB_FUSE_MAXC];
};
struct FusedColPass
{
	int nclass;
	u32 begin[AB_FUSE_MAXC + 1];
	u32 nbx[AB_FUSE_MAXC];        // RC / 32 column groups
	u32 njobs[AB_FUSE_MAXC];
	int sel[AB_FUSE_MAXC];        // LA * 8 + K
	ColJobs jobs[AB_FUSE_MAXC];
};
// Shared memory of the fused row pass for rows of 2^log_r words.
size_t fused_rowpass_smem(int log_r);
// ctas: begin[nclass]; smem: the largest need of the classes.
cudaError_t launch_fused_rowpass(const FusedRowPass * d, const TConst * tcs, u32 ctas, size_t smem, cudaStream_t s);
cudaError_t launch_fused_colpass(const FusedColPass * d, const TConst * tcs, u32 ctas, size_t smem, cudaStream_t s);

// Register words of the reference (K planes of residues mod its primes) from
// the normal form, and back.  The import sets *bad when a coefficient's value
// does not fit the 96-bit normal form (the words are not a normal-form
// register).
cudaError_t launch_export(const RefConst & rc, const u32 * norm, u32 * words, u32 n, cudaStream_t s);
cudaError_t launch_import(const RefConst & rc, const u32 * words, u32 * norm, u32 n, u32 * bad, cudaStream_t s);

} // namespace ab
