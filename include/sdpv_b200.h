/* sdpv_b200 -- B200 (sm_100a) kernels for SDPviBe's multiprecision arithmetic hot path.
 *
 * C ABI of libsdpv_b200.so.  Plain pointers and sizes only: every array argument is a DEVICE pointer
 * on the current CUDA device unless its name ends in `_host`; `stream` is a cudaStream_t (NULL = the
 * legacy default stream).  Every function returns an sdpv_status.  No function allocates device
 * memory except sdpv_ctx_create (its tables, once per limb count and device).
 *
 * Number formats are the reference's:
 *   limb planes   X[k*B + e]: k-th 32-bit limb (little endian, two's complement) of entry e
 *                 (sdpvibe/limbops.py:3-5);
 *   MPF           m (L, n) limb planes + e (n) int64, value = m 2^e, |m| has NB = 32L-2 bits,
 *                 zero is m = 0, e = -2^40 (sdpvibe/mpf.py:1-10, 21);
 *   residues      (G, rows, kp) int8 hi/lo planes, r = 128 hi + lo centred in (-m/2, m/2]
 *                 (sdpvibe/rns.py:196-214);
 *   accumulator   (n, rows, N) int16, canonical residues in [0, m) (sdpvibe/rns.py:106-137).
 *
 * The reference has no C ABI: its Python calls these operations as Triton kernels or CuPy/NVRTC
 * kernels.  Each entry point below names the reference function it replaces (file:line); the
 * Python host layer `sdpvibe_b200` keeps the reference's Python signatures on top of them.
 */
#ifndef SDPV_B200_H
#define SDPV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SDPV_OK = 0,
  SDPV_EOVERFLOW = 1, /* a rounding step overflowed its limb budget (limbops.py:165-185) */
  SDPV_ENOTSPD = 2,   /* non-positive pivot in a Cholesky tile (mpf.py:475-476) */
  SDPV_ETIMEOUT = 3,  /* a bounded device wait gave up (pipeline barrier never completed) */
  SDPV_EINVAL = 4,    /* bad argument (shape, alignment, size beyond a documented limit) */
  SDPV_ECUDA = 5,     /* a CUDA runtime call failed */
  SDPV_ENOMEM = 6     /* table allocation failed */
} sdpv_status;

/* Device error word bits, read (and cleared) by sdpv_get_error. */
#define SDPV_ERRBIT_OVERFLOW 1u
#define SDPV_ERRBIT_TIMEOUT 2u
#define SDPV_ERRBIT_NOTSPD 4u

typedef struct sdpv_ctx sdpv_ctx;

int sdpv_version(void);

/* Last CUDA error text of this thread (for diagnostics after SDPV_ECUDA). */
const char* sdpv_last_error(void);

/* ---------------------------------------------------------------- RNS context
 * Moduli: primes descending from 32639 above 2^14 until M > 4*kmax*2^(2(32L-1)) and n is a multiple
 * of 16 (kmax = 2^17); CRT width E bytes = (ceil(bits(M)/8) + 2 + 7)//8*8, W = E/4 words.
 * Replaces RNS.__init__ (sdpvibe/rns.py:166-191) and mpmat.ctx (sdpvibe/mpmat.py:163-166).
 * Tables live on the device that is current at creation. */
int sdpv_ctx_create(int L, sdpv_ctx** out);
/* The same with the moduli taken in groups of G (1, 2, 4, 8 or 16; sdpv_ctx_create is G = 16, the
 * reference's): the least multiple of G primes that meets the bound.  Replaces the G argument of
 * RNS.__init__ (sdpvibe/rns.py:163-173).  Every G gives the same exact products and CRT values; the
 * autotuner picks it (SDPV_TUNE_MOD_GROUP) for the library's own contexts. */
int sdpv_ctx_create_g(int L, int G, sdpv_ctx** out);
int sdpv_ctx_destroy(sdpv_ctx* ctx);
/* n moduli, E CRT bytes, W = E/4 words. */
int sdpv_ctx_query(const sdpv_ctx* ctx, int* n, int* E, int* W);
/* Copy the n moduli to host memory. */
int sdpv_ctx_moduli(const sdpv_ctx* ctx, int32_t* mods_host);

/* ---------------------------------------------------------------- limb-plane bookkeeping */
/* out = round_half_up(X / 2^s) (ties toward +infinity) as Lout limbs, s per entry (s <= 0: exact
 * left shift).  flag != NULL: per-entry overflow flags (0/1); flag == NULL: overflow sets the
 * device error word.  Replaces limbops.shift_round (sdpvibe/limbops.py:31-62, 173-185). */
int sdpv_shift_round(const int32_t* X, int Lin, int64_t B, const int64_t* s, int Lout, int32_t* out, int32_t* flag,
                     void* stream);
/* out = A + sgn*B mod 2^(32L), sgn = +-1.  Replaces limbops.add_same (sdpvibe/limbops.py:65-81, 188-193). */
int sdpv_add_same(const int32_t* A, const int32_t* Bm, int L, int64_t B, int sgn, int32_t* out, void* stream);
/* out[e] = bit length of v (v >= 0) or of ~v (v < 0).  Replaces limbops.bitlen_words
 * (sdpvibe/limbops.py:196-218). */
int sdpv_bitlen(const int32_t* X, int L, int64_t B, int64_t* out, void* stream);
/* Per entry of (nb, rows, cols): both operands rounded half up to exponent max(ea,eb)+1 of their
 * (block, column), then A + sign*B (wrapping); EO (nb, cols) receives the exponents.
 * Replaces batched.badd(out_exp="align") (sdpvibe/batched.py:55-92). */
int sdpv_badd_align(const int32_t* A, const int32_t* Bm, const int64_t* EA, const int64_t* EB, int L, int64_t nb,
                    int64_t rows, int64_t cols, int sign, int32_t* out, int64_t* EO, void* stream);

/* ---------------------------------------------------------------- per-entry floating point (MPF) */
/* O = A*B entrywise (B a single entry if bscalar), renormalised to NB bits, magnitude rounded half
 * up.  Replaces mpf.mul / mpf_mul (sdpvibe/mpf.py:58-89, 316-323). */
int sdpv_mpf_mul(int L, int64_t n, const int32_t* A, const int64_t* eA, const int32_t* Bm, const int64_t* eB,
                 int bscalar, int32_t* O, int64_t* eO, void* stream);
/* O = A + sgn*B entrywise.  Replaces mpf.add / mpf_add (sdpvibe/mpf.py:92-124, 326-331). */
int sdpv_mpf_add(int L, int64_t n, const int32_t* A, const int64_t* eA, const int32_t* Bm, const int64_t* eB,
                 int sgn, int32_t* O, int64_t* eO, void* stream);
/* ---------------------------------------------------------------- launch-shape knobs (autotuner)
 * Results never depend on them.  SDPV_TUNE_CRT_CTAS: CRT CTAs per SM (1..4, default 3);
 * SDPV_TUNE_NARROW_MAX: residue-GEMM narrow items when one side has at most this many rows (0 = never,
 * else a multiple of 16 up to 64; default 64); SDPV_TUNE_PACK_MAX: small blocks packed several to a tile
 * when both sides have at most this many rows (0 = never, multiple of 16 up to 64; default 64);
 * SDPV_TUNE_RES_WARPS: reducer warps of the decomposition kernel (8 or 16; default 8);
 * SDPV_TUNE_MOD_GROUP: the moduli group G of the contexts the Python layer creates for its own products
 * (1, 2, 4, 8 or 16; default 16; read there, see sdpv_ctx_create_g).
 * No reference counterpart (the reference's launch shapes are fixed). */
#define SDPV_TUNE_CRT_CTAS 0
#define SDPV_TUNE_NARROW_MAX 1
#define SDPV_TUNE_PACK_MAX 2
#define SDPV_TUNE_RES_WARPS 3
#define SDPV_TUNE_MOD_GROUP 4
#define SDPV_TUNE_COUNT 5
int sdpv_tune_set(int knob, int value);
int sdpv_tune_get(int knob, int* value);
/* ---------------------------------------------------------------- binary SDP records (El::BigFloat over GMP limbs)
 * Record: byte is_zero; unless zero, int32 size, int64 exp, nl 64-bit limbs; value = sign(size) M
 * 2^(64 (exp - |size|)).  Replaces decode_bigfloats / encode_bigfloats (sdpvibe/_bigfloat.c:16-111).
 * sdpv_bigfloat_index (host, no launch): offsets of n records from pos; SDPV_EINVAL if truncated/corrupt.
 * sdpv_bigfloat_unpack: device records at offsets -> planar (L, n) limbs + exponents, mantissa rounded half
 *   up to at most 32 L - 2 bits (L <= 64, nl <= 64).
 * sdpv_bigfloat_pack: planar limbs + exponents -> device records at offsets (1 or 13 + 8 nl bytes each);
 *   a mantissa wider than nl limbs sets SDPV_ERRBIT_OVERFLOW. */
int sdpv_bigfloat_index(const uint8_t* buf, int64_t len, int64_t pos, int64_t n, int nl, int64_t* offsets,
                        int64_t* end);
int sdpv_bigfloat_unpack(const uint8_t* buf, const int64_t* offsets, int64_t n, int nl, int L, int32_t* out,
                         int64_t* exps, void* stream);
int sdpv_bigfloat_pack(const int32_t* m, const int64_t* e, int64_t n, int L, int nl, const int64_t* offsets,
                       uint8_t* out, void* stream);
/* Schur complement of one chunk: S (L, nb, P, P) / eS from the pairings AXI, AY (L, 2 nb, W, W) / (2 nb, W, W),
 * W = dim K, P = K dim (dim + 1) / 2, in one launch with the reference's products and sums in its order
 * (bit-exact); S symmetric, diagonal entries of rows with xmask (nb, P, bytes) false set to one_m / one_e
 * (L <= 64).  Replaces the assembly of sdpvibe/solver.py:634-652 (elementwise mpf_mul / mpf_add over
 * sub-blocks, fold over the parities, the 1/4 scale, copy of the lower triangle, padding diagonal). */
int sdpv_schur_assemble(int L, int64_t nb, int P, int K, int dim, const int32_t* AXI, const int64_t* eAXI,
                        const int32_t* AY, const int64_t* eAY, const uint8_t* xmask, const int32_t* one_m,
                        int64_t one_e, int32_t* S, int64_t* eS, void* stream);
/* float64 values V (n) -> normalised MPF (L >= 2 limbs), exactly; zeros -> EZ; a non-finite value
 * becomes zero and sets SDPV_ERRBIT_OVERFLOW.  Replaces the host frexp conversion of
 * sdpvibe/solver.py:1012-1018 (the float64 -> mpf step of the step-length code). */
int sdpv_mpf_from_f64(int L, int64_t n, const double* V, int32_t* O, int64_t* eO, void* stream);
/* Normalise LI-limb integers with exponents eI to MPF with L limbs (LI <= 160).
 * Replaces mpf.normalize / mpf_norm (sdpvibe/mpf.py:127-140, 307-313). */
int sdpv_mpf_norm(int L, int LI, int64_t n, const int32_t* X, const int64_t* eI, int32_t* O, int64_t* eO,
                  void* stream);

/* ---------------------------------------------------------------- operand alignment
 * MPF array m (L, nb, R, C) / e (nb, R, C).  top = e + bitlen(m), EZ for zero entries.
 * axis 1: out (nb, R) = max over columns of each row; axis 0: out (nb, C) = max over rows of each column.
 * Replaces _top(A).amax(...) (sdpvibe/mpf.py:348-351, 393, 563). */
int sdpv_top_max(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C, int axis, int64_t* out,
                 void* stream);
/* out = m rounded half up (ties toward +infinity) to the exponent target[b][r] (per_col = 0) or target[b][c]
 * (per_col = 1), as Lout limbs; zero entries (e = EZ) become 0; transpose = 1 writes (Lout, nb, C, R) instead of
 * (Lout, nb, R, C).  Overflow sets the device error word.  L <= 64.  Replaces the transposing copy plus
 * shift_round of mpf._align_rows (sdpvibe/mpf.py:390-398) and GramAcc.add (sdpvibe/mpf.py:572-576). */
int sdpv_align(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C, const int64_t* target,
               int per_col, int transpose, int Lout, int32_t* out, void* stream);
/* sdpv_align with transpose = 1 into (Lout, nb, C, Rld) limb planes, Rld >= R (rows R .. Rld - 1 of each
 * column are left untouched): a row length that is a multiple of 4 lets the decomposition read the planes
 * with bulk tensor copies.  No reference counterpart. */
int sdpv_align_t(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C, const int64_t* target,
                 int per_col, int Lout, int64_t Rld, int32_t* out, void* stream);
/* The transposed alignment written as operand rows for sdpv_residues_rows: entry (b, r, c) of m becomes row
 * (b C + c) Rp + r of out (nb, C, Rp, rb) uint8, rb = 128 bytes for Lout <= 31, 256 for Lout <= 63: the Lout
 * aligned limbs little endian, then a sign byte (1 when the result is negative) at byte 4 Lout, then zeros;
 * rows R .. Rp - 1 of each column are zero rows.  Rp >= R, a multiple of 128.  Same rounding and overflow
 * rule as sdpv_align.  No reference counterpart (an internal layout of GramAcc.add's aligned chunk). */
int sdpv_align_rows(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C,
                    const int64_t* target, int per_col, int Lout, int64_t Rp, uint8_t* out, void* stream);

/* ---------------------------------------------------------------- residue decomposition (a)
 * Residues of X[:, :, k0:k0+kc] for moduli g0..g0+G of ctx: X (L, rows, ld) int32 limb planes;
 * Rhi, Rlo (G, rows, kp) int8, kp = kc rounded up to 16, zero residues for kc <= k < kp; plane_stride = bytes
 * between the planes of consecutive moduli (0: rows*kp, contiguous; otherwise a multiple of 16 >= rows*kp --
 * an odd multiple of 2 KB keeps the 2G concurrent plane streams on different HBM channels).
 * Replaces RNS.residues / _residue_kernel (sdpvibe/rns.py:66-103, 196-214). */
int sdpv_residues(const sdpv_ctx* ctx, const int32_t* X, int64_t rows, int64_t ld, int64_t k0, int64_t kc, int g0,
                  int G, int8_t* Rhi, int8_t* Rlo, int64_t plane_stride, void* stream);
/* The same decomposition in the GEMM's internal digit format: the canonical residue r in [0, m) as
 * Rhi = r >> 7 in [0, 256), Rlo = r & 127 (uint8), for sdpv_rns_gemm with mode bit 2.  No reference
 * counterpart (an internal format: one centring correction less per residue). */
int sdpv_residues_u8(const sdpv_ctx* ctx, const int32_t* X, int64_t rows, int64_t ld, int64_t k0, int64_t kc, int g0,
                     int G, uint8_t* Rhi, uint8_t* Rlo, int64_t plane_stride, void* stream);
/* sdpv_residues_u8 of operand rows (sdpv_align_rows, ctx's L limbs): entry (i, k) of the result (i < nI,
 * k < kc) is row i Rp + k0 + k of rows.  k0 and Rp multiples of 128, k0 + kc <= Rp, rows k0 + kc .. k0 + kp - 1
 * zero (so when kc is not a multiple of 16, k0 + kc must be the column's row count); g0 a multiple of 128;
 * ctx's L <= 63.  Rhi, Rlo (G, nI, kp) as sdpv_residues_u8. */
int sdpv_residues_rows(const sdpv_ctx* ctx, const uint8_t* rows, int64_t nI, int64_t Rp, int64_t k0, int64_t kc,
                       int g0, int G, uint8_t* Rhi, uint8_t* Rlo, int64_t plane_stride, void* stream);

/* ---------------------------------------------------------------- residue GEMM (b) and Gram (d)
 * For each of the G moduli g0..g0+G and each of nb blocks:
 *   acc[g0+g][b*M + i][j] <- (acc + A_gb B_gb^T) mod m, A_gb = 128 Ahi + Alo (M x KC), B likewise (N x KC)
 * with A* (G, nb*M, KC), B* (G, nb*N, KC) int8 whose modulus planes are a_stride / b_stride bytes apart (0: packed),
 * acc (n, nb*M, ldc) int16 (row stride ldc >= N; a
 * multiple of 8 lets the epilogue move 16 bytes at a time).  mode bit 0 clear: all entries;
 * set (syrk): B = A (Bhi/Blo ignored, N = M) and only entries with i >= j are updated.  mode bit 1 set
 * (fresh): the updated entries of acc are taken as zero and overwritten, not read.  mode bit 2 set: the
 * operands are unsigned digits (sdpv_residues_u8; KC <= 32768 keeps the int32 sums exact).
 * KC must be a multiple of 16 and <= 65536.  Replaces RNS.accumulate / _gemm_kernel
 * (sdpvibe/rns.py:106-137, 217-224), batched._bgemm_kernel (sdpvibe/batched.py:96-127) and
 * batched._syrk_lower_kernel (sdpvibe/batched.py:130-162). */
int sdpv_rns_gemm(const sdpv_ctx* ctx, const int8_t* Ahi, const int8_t* Alo, const int8_t* Bhi, const int8_t* Blo,
                  int64_t a_stride, int64_t b_stride, int16_t* acc, int64_t ldc, int g0, int G, int64_t nb, int64_t M, int64_t N, int64_t KC, int mode, void* stream);

/* ---------------------------------------------------------------- CRT reconstruction (c)
 * Exact integers of the block "all rows x columns j0..j0+w" of acc (n, rows_total, N) (modulus
 * stride ldg entries): words (W, rows*w) int32 two's complement (entry e = i*w + jj) and bit lengths
 * (rows*w) of v / ~v.  Valid for |value| < M/4.  Replaces RNS.crt_block with crt_pre / crt dot /
 * crt_carry (sdpvibe/rns.py:140-159, 227-245; sdpvibe/limbops.py:85-152, 221-239). */
int sdpv_crt_block(const sdpv_ctx* ctx, const int16_t* acc, int64_t ldg, int64_t N, int64_t j0, int64_t w,
                   int64_t rows, int32_t* words, int64_t* bitlen, void* stream);

/* CRT fused with renormalisation to MPF (mpf_norm semantics): for the same block, entry (r, jj) with
 * exponent rowexp[r] + colexp[(r / rows_per_block) * N + j0 + jj] is written to O (L, rows*w) /
 * eO (rows*w).  Replaces the crt_block + normalize pairs of mpf.gemm (sdpvibe/mpf.py:440-450) and
 * GramAcc._crt (sdpvibe/mpf.py:595-610). */
int sdpv_crt_norm(const sdpv_ctx* ctx, const int16_t* acc, int64_t ldg, int64_t N, int64_t j0, int64_t w,
                  int64_t rows, int64_t rows_per_block, const int64_t* rowexp, const int64_t* colexp, int L,
                  int32_t* O, int64_t* eO, void* stream);

/* ---------------------------------------------------------------- Cholesky base case (e)
 * Wide fixed point: a tile entry is WL 32-bit words (two's complement) with F = 32*LF fraction bits;
 * tiles are entry-major (ntiles, 32, 32, WL); bt must be 32; WL <= 96.
 * sdpv_chol_tiles: in-place lower Cholesky of each tile (upper part untouched) and the pivot reciprocals
 * RINV (ntiles, 32, WL); a non-positive pivot sets SDPV_ERRBIT_NOTSPD in the device error word.
 * Replaces chol_tiles (sdpvibe/basecase.py:158-193). */
int sdpv_chol_tiles(uint32_t* A, uint32_t* RINV, int64_t ntiles, int bt, int WL, int LF, void* stream);
/* X = L^-1 of lower tiles whose upper part is zero; S: caller workspace of the same size as X.
 * Replaces trinv_tiles (sdpvibe/basecase.py:195-226). */
int sdpv_trinv_tiles(const uint32_t* Lt, const uint32_t* RINV, uint32_t* X, uint32_t* S, int64_t ntiles, int bt,
                     int WL, int LF, void* stream);

/* sdpv_mpf_add that runs only if *pred (a device int32) is nonzero; O may alias A (in-place accumulation).
 * With sdpv_crt_norm_if it lets GramAcc add a flushed partial sum without a host decision
 * (sdpvibe/mpf.py:612-616). */
/* One Gram chunk's column bookkeeping on the device (GramAcc.add, sdpvibe/mpf.py:556-579): from the chunk's
 * column tops tp (N), updates the reference exponents E and the running tops Tmax in place, writes the flush
 * predicate *f (some seen column outgrew E by more than head bits), the flush's CRT exponents rE_old (E - nbits
 * before the update, 0 for unseen columns), the chunk's alignment targets (E - nbits after it), and adds *f to
 * *nflush when has_acc.  One launch instead of the elementwise sequence. */
int sdpv_gram_columns(int64_t N, const int64_t* tp, int64_t* E, int64_t* Tmax, int64_t head, int64_t nbits, int has_acc,
                      int64_t* rE_old, int64_t* target, int32_t* f, int64_t* nflush, void* stream);
/* Zeroes nbytes (a multiple of 16, 16-byte aligned) at p when *pred (a device int32) is nonzero: the Gram
 * accumulator after a flush, decided on the device. */
int sdpv_zero_if(void* p, int64_t nbytes, const int32_t* pred, void* stream);
int sdpv_mpf_add_if(int L, int64_t n, const int32_t* A, const int64_t* eA, const int32_t* Bm, const int64_t* eB,
                    int sgn, int32_t* O, int64_t* eO, const int32_t* pred, void* stream);

/* sdpv_crt_norm that runs only if *pred (a device int32) is nonzero, so that a caller can decide on the device
 * whether a partial Gram sum must be reconstructed (GramAcc's flush, sdpvibe/mpf.py:557-616) without a host
 * synchronisation.  When *pred is zero, O and eO are left untouched. */
int sdpv_crt_norm_if(const sdpv_ctx* ctx, const int16_t* acc, int64_t ldg, int64_t N, int64_t j0, int64_t w,
                     int64_t rows, int64_t rows_per_block, const int64_t* rowexp, const int64_t* colexp, int L,
                     int32_t* O, int64_t* eO, const int32_t* pred, void* stream);

/* Eigenvalues of nb symmetric float64 n x n matrices A (nb, n, n) (n <= 128), ascending into w (nb, n), with an
 * error bound per matrix in err (nb) and the sweep count in sweeps (nb, may be NULL): batched cyclic Jacobi.
 * The device counterpart of the host LAPACK call in the step length (sdpvibe/solver.py:1064-1093, the
 * eigvalsh of the scaled float64 copy, and _eig_err 1001-1004). */
int sdpv_eig_sym_f64(const double* A, int64_t nb, int n, double* w, double* err, int* sweeps, void* stream);

/* Triangular solve L y = v for nvec vectors of 32 entries with one factored 32 x 32 tile (Lt lower, RINV its
 * pivot reciprocals), wide fixed point; V (nvec, 32, WL) is overwritten by y.  Replaces basecase.trsv_tile's
 * trsv_warp (sdpvibe/basecase.py:228-245, 310-331). */
int sdpv_trsv_tiles(const uint32_t* Lt, const uint32_t* RINV, uint32_t* V, int64_t nvec, int bt, int WL, int LF,
                    void* stream);

/* Allocation-free sdpv_trinv_tiles, for callers that cannot allocate device memory at the point of the call
 * (their process has handed all device memory to another allocator, or the calling code must not allocate).
 * No counterpart in the reference.  For WL <= 64 the inverse runs in shared memory and uses no scratch, at
 * any ntiles.  For WL > 64 the product scratch is a fixed 16 MiB array inside the library image (4 Mi 32-bit
 * words): the call needs ntiles * 32 * 32 * WL <= 4 Mi words and returns SDPV_EINVAL beyond that.  The array
 * is held on a device from the moment the library's tile module is loaded there -- with lazy module loading
 * (the CUDA 12 default) at the first call of any tile entry point (sdpv_chol_tiles, sdpv_trinv_tiles,
 * sdpv_trsv_tiles, this one) on that device -- until the process exits; make that first call before handing
 * device memory to another allocator, and before any stream capture (it also looks up the array's device
 * address).  All calls on a device share the array: calls with WL > 64 that overlap on the GPU (different
 * streams, no ordering) race on it.  Nothing in the array needs to start at zero; every word a call reads was
 * written earlier in the same call. */
int sdpv_trinv_tiles_noalloc(const uint32_t* Lt, const uint32_t* RINV, uint32_t* X, int64_t ntiles, int bt, int WL,
                             int LF, void* stream);

/* ---------------------------------------------------------------- grouped Cholesky / triangular solves
 * The batched Cholesky factorisation and triangular solves of blocks of different sizes run as waves over a
 * device work list (the host plan of sdpvibe_b200/grouped.py): every entry point below takes a device table
 * of descriptors whose rows may belong to blocks of any size, so one launch serves all blocks of a wave.
 * Together they replace the reference's per-bucket recursion bchol / btrsm_right / btrsm_left /
 * btrsm_left_T (sdpvibe/batched.py:243-352, called per padded block size by mpf.Chol, sdpvibe/mpf.py:461-532)
 * with results identical block by block.  Arenas are limb planes (plane stride = entries per plane):
 * factor tiles (L, T, 32, 32), tile inverses (L, D, 32, 32) with exponents xe (D), solve row tiles
 * (L, RT, 32, m) with exponents Pe (RT, m).
 *
 * Grouped narrow residue products (the work-list form of sdpv_rns_gemm): items (8 int32 each: big-side row0,
 * big rows <= 128, small-side row0, small rows <= TB, K length (multiple of 32, <= KP), output row0, output
 * column0, 0) multiply rows of the big side (unsigned residue digits, (G, big_rows, KP) planes big_stride
 * bytes apart) against rows of the small side over their own K; out_mode 1 stores acc[g][out_row0 + r][j],
 * out_mode 2 acc[g][out_row0 + j][out_col0 + r] (acc (n, rows_out, ldc) int16, fresh).  TB in 16..64,
 * multiple of 16. */
int sdpv_rns_gemm_grouped(const sdpv_ctx* ctx, const uint8_t* bigHi, const uint8_t* bigLo, int64_t big_rows,
                          int64_t big_stride, const uint8_t* smallHi, const uint8_t* smallLo, int64_t small_rows,
                          int64_t small_stride, int64_t KP, int TB, int out_mode, const int32_t* items, int64_t nitems,
                          int16_t* acc, int64_t ldc, int64_t rows_out, int g0, int G, void* stream);

/* Block copies into a workspace (L, ., .): desc (8 int64 each: source arena, source base entry, source row
 * stride, destination base entry, destination row stride, rows <= 32, cols <= 32, transpose); src_host /
 * src_planes_host: HOST arrays of nsrc (<= 4) arena device pointers and their plane strides. */
int sdpv_grp_copy(int32_t* const* src_host, const int64_t* src_planes_host, int nsrc, int32_t* dst, int64_t dst_plane,
                  int L, const int64_t* desc, int64_t ndesc, void* stream);

/* Fixed-exponent rounding of CRT words (W words, planes Ntot apart, entry = row * w + column) combined into
 * arena blocks: desc (40 int64 each: out arena, out base, out ld, base arena or -1, base base, base ld, rows,
 * cols, nsrc <= 7, then per source CRT entry base, sign, shift constant, exponent index or -1):
 * out = base + sum sign round(W / 2^(cst - xe[idx])) mod 2^(32L) -- btrsm_right's and bchol's rounded
 * products and exact differences (sdpvibe/batched.py:274-305, 82-92). */
int sdpv_grp_finish_fixed(const int32_t* Wd, int W, int64_t Ntot, int64_t w, int32_t* const* ar_host,
                          const int64_t* planes_host, int nar, int L, const int64_t* xe, const int64_t* desc,
                          int64_t ndesc, void* stream);

/* Per-column ('col') rounding of a group of solve outputs: desc (10 int64 each: CRT row0, rows, column0,
 * ncols <= 32, eA constant, eA index or -1, B row tile, mode, base row tile0, destination row tile0); the
 * group's column exponent from its rows' maximal bit length, then store (mode 0) or the aligned difference /
 * sum with the base rows (modes 1 / 2) -- btrsm_left's leaf, update and badd 'align' (sdpvibe/batched.py:
 * 200-231, 313-352, 55-92). */
int sdpv_grp_solve_round(const int32_t* Wd, const int64_t* bl, int W, int64_t Ntot, int64_t w, int32_t* P,
                         int64_t Pplane, int64_t* Pe, int64_t m, int L, const int64_t* xe, const int64_t* desc,
                         int64_t ndesc, void* stream);

/* Common column exponents of a tree node's row tiles: desc (4 int64 each: row tile0, row tiles, column0,
 * ncols <= 32); both halves re-rounded to the larger exponent (sdpvibe/batched.py:332-335, 349-352). */
int sdpv_grp_merge(int32_t* P, int64_t Pplane, int64_t* Pe, int64_t m, int L, const int64_t* desc, int64_t ndesc,
                   void* stream);

/* Diagonal tiles of the factor arena (entry bases fbase, exponent e) -> wide fixed point (ntiles, 32, 32, WL)
 * at exponent -32 LF, zero above the diagonal (sdpvibe/batched.py:250). */
int sdpv_grp_tile_widen(const int32_t* Fa, int64_t Fplane, int L, int64_t e, int WL, int LF, const int64_t* fbase,
                        int64_t ntiles, uint32_t* out, void* stream);

/* Factored wide tiles (Lw) and their inverses (Xw) back to the arenas: the factor at e (zero above the
 * diagonal), the inverse at xe[xidx] = max bit length - 32 LF - (32 L - 32) per tile (sdpvibe/batched.py:
 * 256-262). */
int sdpv_grp_tile_narrow(const uint32_t* Lw, const uint32_t* Xw, int WL, int LF, int32_t* Fa, int64_t Fplane, int L,
                         int64_t e, const int64_t* fbase, int32_t* Xa, int64_t Xplane, const int64_t* xidx,
                         int64_t* xe, int64_t ntiles, void* stream);

/* ---------------------------------------------------------------- errors
 * Read and clear the device error word (bits SDPV_ERRBIT_*) after synchronising `stream`.
 * Replaces limbops.check_errors (sdpvibe/limbops.py:156-169). */
int sdpv_get_error(unsigned* flags_host, void* stream);

/* Synchronise `stream`, read and clear the device error word, and return it as a status: SDPV_ETIMEOUT when a
 * bounded device wait gave up, else SDPV_ENOTSPD, else SDPV_EOVERFLOW, else SDPV_OK.  The status form of
 * limbops.check_errors (sdpvibe/limbops.py:156-169) that also reports the pipelines' wait timeouts. */
int sdpv_device_status(void* stream);

/* Launch one warp that waits on a shared-memory barrier with the pipelines' bounded wait, its limit shortened
 * to limit_us microseconds (1 .. 2e6).  arrive != 0: the barrier completes and the wait returns at once;
 * arrive == 0: nothing completes it, so the wait gives up after limit_us, sets SDPV_ERRBIT_TIMEOUT and the
 * kernel returns (the context stays usable); sdpv_device_status then reports SDPV_ETIMEOUT.  Exercises the
 * timeout path of every pipeline wait.  No counterpart in the reference (its kernels have no bounded waits). */
int sdpv_wait_probe(unsigned limit_us, int arrive, void* stream);

#ifdef __cplusplus
}
#endif
#endif
