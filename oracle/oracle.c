/* CPU oracle for the multiprecision hot path -- TEST INFRASTRUCTURE ONLY (the checker, never the
 * product).  Plain C restatement of SDPviBe's integer arithmetic, one function per reference kernel,
 * each citing the file:line it follows.  Layout conventions are the reference's: a batch of B
 * multiword integers is stored as limb planes X[k*B + e] (k-th 32-bit limb, little endian, two's
 * complement); wide fixed-point tiles of the Cholesky base case are entry-major (AoS) words.
 *
 * Built by oracle/Makefile into oracle/liboracle.so and driven from oracle/__init__.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;

#define MASK32 0xffffffffULL
static const i64 EZ = -(1LL << 40); /* exponent of zero, sdpvibe/mpf.py:21 */

/* ---------------------------------------------------------------- limb-plane bookkeeping */

/* Word i of the two's-complement extension of X (sign-extended above, zero below). */
static inline u64 word_at(const int32_t* X, int L, i64 B, i64 e, i64 i, u64 ext) {
  if (i < 0) return 0;
  if (i >= L) return ext;
  return (u64)(u32)X[i * B + e];
}

/* Bits [32q + r, 32q + r + 32) of X (r in [0, 32)): limbops.py:21-28. */
static inline u64 window(const int32_t* X, int L, i64 B, i64 e, i64 q, int r, u64 ext) {
  u64 lo = word_at(X, L, B, e, q, ext), hi = word_at(X, L, B, e, q + 1, ext);
  return ((lo | (hi << 32)) >> r) & MASK32;
}

static inline i64 floordiv32(i64 s) { return s >> 5; } /* arithmetic shift = floor division */

/* round_half_up(X / 2^s) to Lout limbs, overflow flag per entry: limbops.py:31-62, 173-185. */
void or_shift_round(const int32_t* X, int Lin, i64 B, const i64* S, int Lout, int32_t* out, int32_t* flag) {
  for (i64 e = 0; e < B; e++) {
    i64 s = S[e];
    i64 q = floordiv32(s);
    int r = (int)(s - 32 * q);
    u64 ext = (X[(i64)(Lin - 1) * B + e] < 0) ? MASK32 : 0;
    i64 sb = s - 1, qb = floordiv32(sb);
    int rb = (int)(sb - 32 * qb);
    u64 carry = (sb >= 0) ? ((word_at(X, Lin, B, e, qb, ext) >> rb) & 1) : 0;
    u64 prev = 0;
    int bad = 0;
    for (int k = 0; k <= Lout; k++) {
      u64 v = window(X, Lin, B, e, q + k, r, ext) + carry;
      carry = v >> 32;
      v &= MASK32;
      if (k < Lout) {
        out[(i64)k * B + e] = (int32_t)(u32)v;
        prev = v;
      } else {
        u64 want = (prev >> 31) ? MASK32 : 0;
        bad = (v != want);
      }
    }
    if (flag) flag[e] = bad;
  }
}

/* A + sgn*B modulo 2^(32L): limbops.py:65-81, 188-193. */
void or_add_same(const int32_t* A, const int32_t* Bm, int L, i64 B, int sgn, int32_t* out) {
  for (i64 e = 0; e < B; e++) {
    i64 carry = 0;
    for (int k = 0; k < L; k++) {
      i64 a = (k == L - 1) ? (i64)A[(i64)k * B + e] : (i64)(u32)A[(i64)k * B + e];
      i64 b = (k == L - 1) ? (i64)Bm[(i64)k * B + e] : (i64)(u32)Bm[(i64)k * B + e];
      i64 v = a + sgn * b + carry;
      carry = v >> 32;
      out[(i64)k * B + e] = (int32_t)(u32)(v & (i64)MASK32);
    }
  }
}

static inline int bitlen32(u32 x) { return x ? 32 - __builtin_clz(x) : 0; }

/* Bit length of v (v >= 0) or of ~v (v < 0): limbops.py:196-218. */
void or_bitlen(const int32_t* X, int L, i64 B, i64* out) {
  for (i64 e = 0; e < B; e++) {
    u32 ext = (X[(i64)(L - 1) * B + e] < 0) ? 0xffffffffu : 0;
    i64 bl = 0;
    for (int k = L - 1; k >= 0; k--) {
      u32 x = (u32)X[(i64)k * B + e] ^ ext;
      if (x) { bl = 32 * (i64)k + bitlen32(x); break; }
    }
    out[e] = bl;
  }
}

/* Aligned batched add: both operands independently rounded (half up) to exponent max(ea,eb)+1,
 * then A + sign*B wrapping to L limbs: batched.py:55-92. */
void or_badd_align(const int32_t* A, const int32_t* Bm, const i64* EA, const i64* EB, int L, i64 nb, i64 rows,
                   i64 cols, int sign, int32_t* out, i64* EO) {
  i64 n = nb * rows * cols;
  for (i64 e = 0; e < n; e++) {
    i64 col = (e / (rows * cols)) * cols + e % cols;
    i64 ea = EA[col], eb = EB[col];
    i64 ex = (ea > eb ? ea : eb) + 1;
    i64 sa = ex - ea, sb = ex - eb;
    u64 ax = (A[(i64)(L - 1) * n + e] < 0) ? MASK32 : 0;
    u64 bx = (Bm[(i64)(L - 1) * n + e] < 0) ? MASK32 : 0;
    i64 qa = floordiv32(sa), qb = floordiv32(sb);
    int ra = (int)(sa - 32 * qa), rb = (int)(sb - 32 * qb);
    i64 qa1 = floordiv32(sa - 1), qb1 = floordiv32(sb - 1);
    u64 ca = window(A, L, n, e, qa1, (int)(sa - 1 - 32 * qa1), ax) & 1;
    u64 cb = window(Bm, L, n, e, qb1, (int)(sb - 1 - 32 * qb1), bx) & 1;
    i64 carry = 0;
    for (int k = 0; k < L; k++) {
      u64 a = window(A, L, n, e, qa + k, ra, ax) + ca;
      u64 b = window(Bm, L, n, e, qb + k, rb, bx) + cb;
      ca = a >> 32;
      cb = b >> 32;
      i64 t = (i64)(a & MASK32) + sign * (i64)(b & MASK32) + carry;
      carry = t >> 32;
      out[(i64)k * n + e] = (int32_t)(u32)(t & (i64)MASK32);
    }
    if ((e / cols) % rows == 0) EO[col] = ex;
  }
}

/* ---------------------------------------------------------------- per-entry floating point (MPF) */
/* Magnitude helpers on little-endian u32 words. */
static void neg_words(u32* a, int n) {
  u64 c = 1;
  for (int k = 0; k < n; k++) {
    u64 t = (u64)(u32)~a[k] + c;
    a[k] = (u32)t;
    c = t >> 32;
  }
}

static int bitlen_words_mag(const u32* a, int n) {
  for (int k = n - 1; k >= 0; k--)
    if (a[k]) return 32 * k + bitlen32(a[k]);
  return 0;
}

/* dst (nd words) = round_half_up(src / 2^s) of a magnitude for s > 0 (carry kept inside nd words),
 * src * 2^-s truncated to nd words for s <= 0: mpf.py:36-56. */
static void mag_shift(const u32* src, int ns, int s, u32* dst, int nd) {
  if (s > 0) {
    int q = s >> 5, r = s & 31;
    for (int k = 0; k < nd; k++) {
      u64 lo = (q + k < ns) ? src[q + k] : 0, hi = (q + k + 1 < ns) ? src[q + k + 1] : 0;
      dst[k] = (u32)(((hi << 32) | lo) >> r);
    }
    int qb = (s - 1) >> 5, rb = (s - 1) & 31;
    u64 c = (qb < ns) ? ((src[qb] >> rb) & 1u) : 0;
    for (int k = 0; k < nd && c; k++) {
      u64 t = (u64)dst[k] + c;
      dst[k] = (u32)t;
      c = t >> 32;
    }
  } else {
    int t = -s, q = t >> 5, r = t & 31;
    for (int k = 0; k < nd; k++) {
      int i0 = k - q, i1 = k - q - 1;
      u64 lo = (i0 >= 0 && i0 < ns) ? src[i0] : 0, lo2 = (i1 >= 0 && i1 < ns) ? src[i1] : 0;
      dst[k] = (u32)((((lo << 32) | lo2) << r) >> 32);
    }
  }
}

#define MPF_MAXW 512

/* Entrywise product, renormalised to NB = 32L-2 bits, magnitude rounded half up: mpf.py:58-89. */
void or_mpf_mul(int L, i64 n, const int32_t* A, const i64* eA, const int32_t* Bv, const i64* eB, int bscalar,
                int32_t* O, i64* eO) {
  int NB = 32 * L - 2;
  i64 nbn = bscalar ? 1 : n;
  for (i64 i = 0; i < n; i++) {
    i64 ib = bscalar ? 0 : i;
    u32 a[MPF_MAXW], b[MPF_MAXW], p[2 * MPF_MAXW], r[MPF_MAXW];
    for (int k = 0; k < L; k++) {
      a[k] = (u32)A[(i64)k * n + i];
      b[k] = (u32)Bv[(i64)k * nbn + ib];
    }
    int na = a[L - 1] >> 31, nb = b[L - 1] >> 31;
    if (na) neg_words(a, L);
    if (nb) neg_words(b, L);
    if (!bitlen_words_mag(a, L) || !bitlen_words_mag(b, L)) {
      for (int k = 0; k < L; k++) O[(i64)k * n + i] = 0;
      eO[i] = EZ;
      continue;
    }
    memset(p, 0, sizeof(u32) * 2 * L);
    for (int x = 0; x < L; x++) { /* operand scanning */
      u64 c = 0;
      for (int y = 0; y < L; y++) {
        u64 t = (u64)a[x] * b[y] + p[x + y] + c;
        p[x + y] = (u32)t;
        c = t >> 32;
      }
      p[x + L] = (u32)c;
    }
    int s = bitlen_words_mag(p, 2 * L) - NB;
    mag_shift(p, 2 * L, s, r, L);
    if (na != nb) neg_words(r, L);
    for (int k = 0; k < L; k++) O[(i64)k * n + i] = (int32_t)r[k];
    eO[i] = eA[i] + eB[ib] + s;
  }
}

/* Entrywise A + sgn*B via an L+2-word common format at exponent max(ea,eb)-32, then
 * renormalised: mpf.py:92-124. */
void or_mpf_add(int L, i64 n, const int32_t* A, const i64* eA, const int32_t* Bv, const i64* eB, int sgn,
                int32_t* O, i64* eO) {
  int NB = 32 * L - 2;
  int far = 32 * (L + 3);
  for (i64 i = 0; i < n; i++) {
    u32 a[MPF_MAXW], b[MPF_MAXW], wa[MPF_MAXW + 2], wb[MPF_MAXW + 2], r[MPF_MAXW];
    for (int k = 0; k < L; k++) {
      a[k] = (u32)A[(i64)k * n + i];
      b[k] = (u32)Bv[(i64)k * n + i];
    }
    int na = a[L - 1] >> 31;
    int nbs = (b[L - 1] >> 31) ^ (sgn < 0);
    if (a[L - 1] >> 31) neg_words(a, L);
    if (b[L - 1] >> 31) neg_words(b, L);
    i64 ea = eA[i], eb = eB[i];
    if (!bitlen_words_mag(a, L)) ea = EZ;
    if (!bitlen_words_mag(b, L)) eb = EZ;
    if (ea == EZ && eb == EZ) {
      for (int k = 0; k < L; k++) O[(i64)k * n + i] = 0;
      eO[i] = EZ;
      continue;
    }
    i64 t = (ea > eb ? ea : eb) - 32;
    i64 da = ea - t, db = eb - t;
    int sa = (da < -(i64)far) ? far : (int)(-da);
    int sb = (db < -(i64)far) ? far : (int)(-db);
    if (ea == EZ) memset(wa, 0, sizeof(u32) * (L + 2)); else mag_shift(a, L, sa, wa, L + 2);
    if (eb == EZ) memset(wb, 0, sizeof(u32) * (L + 2)); else mag_shift(b, L, sb, wb, L + 2);
    if (na) neg_words(wa, L + 2);
    if (nbs) neg_words(wb, L + 2);
    u64 c = 0;
    for (int k = 0; k < L + 2; k++) {
      u64 v = (u64)wa[k] + wb[k] + c;
      wa[k] = (u32)v;
      c = v >> 32;
    }
    int ns = wa[L + 1] >> 31;
    if (ns) neg_words(wa, L + 2);
    int bl = bitlen_words_mag(wa, L + 2);
    if (!bl) {
      for (int k = 0; k < L; k++) O[(i64)k * n + i] = 0;
      eO[i] = EZ;
      continue;
    }
    int s = bl - NB;
    mag_shift(wa, L + 2, s, r, L);
    if (ns) neg_words(r, L);
    for (int k = 0; k < L; k++) O[(i64)k * n + i] = (int32_t)r[k];
    eO[i] = t + s;
  }
}

/* Normalise LI-limb two's-complement integers with exponents eI to L limbs: mpf.py:127-140. */
void or_mpf_norm(int L, int LI, i64 n, const int32_t* X, const i64* eI, int32_t* O, i64* eO) {
  int NB = 32 * L - 2;
  for (i64 i = 0; i < n; i++) {
    u32 w[MPF_MAXW], r[MPF_MAXW];
    for (int k = 0; k < LI; k++) w[k] = (u32)X[(i64)k * n + i];
    int ng = w[LI - 1] >> 31;
    if (ng) neg_words(w, LI);
    int bl = bitlen_words_mag(w, LI);
    if (!bl) {
      for (int k = 0; k < L; k++) O[(i64)k * n + i] = 0;
      eO[i] = EZ;
      continue;
    }
    int s = bl - NB;
    mag_shift(w, LI, s, r, L);
    if (ng) neg_words(r, L);
    for (int k = 0; k < L; k++) O[(i64)k * n + i] = (int32_t)r[k];
    eO[i] = eI[i] + s;
  }
}

/* ---------------------------------------------------------------- residue number system */

/* Residues of X[:, :, k0:k0+kc] (L, rows, ld) modulo mods[0..G), centred to (-m/2, m/2] and split
 * r = 128*hi + lo, lo in [-64, 64); columns kc <= k < kp are residues of zero: rns.py:66-103,196-214. */
struct res_job {
  const int32_t* X;
  int L, G, nthr, t;
  i64 rows, ld, k0, kc, kp;
  const int32_t* mods;
  int8_t *Rhi, *Rlo;
};

/* Moduli t, t + nthr, ... of one or_residues call.  Per row, Horner over the limbs (most significant first,
 * the top limb signed) on all kc entries of the row at once, so each limb row is read sequentially.
 * |r| < m < 2^15 and 2^32 mod m < 2^15, so r * w32 + v stays inside int64 and one remainder per limb
 * suffices. */
static void* res_worker(void* arg) {
  const struct res_job* J = (const struct res_job*)arg;
  i64 plane = J->rows * J->ld, kc = J->kc, kp = J->kp;
  i64* r = (i64*)malloc(sizeof(i64) * (size_t)(kc > 0 ? kc : 1));
  for (int g = J->t; g < J->G; g += J->nthr) {
    i64 m = J->mods[g];
    i64 w32 = (i64)(((u64)1 << 32) % (u64)m); /* 2^32 mod m */
    for (i64 i = 0; i < J->rows; i++) {
      for (i64 k = 0; k < kc; k++) r[k] = 0;
      for (int l = J->L - 1; l >= 0; l--) {
        const int32_t* x = J->X + l * plane + i * J->ld + J->k0;
        if (l == J->L - 1)
          for (i64 k = 0; k < kc; k++) r[k] = (r[k] * w32 + (i64)x[k]) % m;
        else
          for (i64 k = 0; k < kc; k++) r[k] = (r[k] * w32 + (i64)(u32)x[k]) % m;
      }
      for (i64 k = 0; k < kp; k++) {
        i64 v = 0;
        if (k < kc) {
          v = r[k];
          if (v < 0) v += m;
        }
        if (v > m / 2) v -= m;
        i64 lo = ((v + 64) & 127) - 64;
        i64 hi = (v - lo) >> 7;
        i64 o = ((i64)g * J->rows + i) * kp + k;
        J->Rhi[o] = (int8_t)hi;
        J->Rlo[o] = (int8_t)lo;
      }
    }
  }
  free(r);
  return NULL;
}

void or_residues(const int32_t* X, int L, i64 rows, i64 ld, i64 k0, i64 kc, i64 kp, const int32_t* mods, int G,
                 int8_t* Rhi, int8_t* Rlo) {
  long nc = sysconf(_SC_NPROCESSORS_ONLN);
  int nthr = (int)(nc < 1 ? 1 : (nc > 64 ? 64 : nc));
  if (nthr > G) nthr = G > 0 ? G : 1;
  if (rows * kc < 4096) nthr = 1;
  struct res_job J[64];
  pthread_t th[64];
  for (int t = 0; t < nthr; t++) {
    J[t] = (struct res_job){X, L, G, nthr, t, rows, ld, k0, kc, kp, mods, Rhi, Rlo};
    if (t > 0) pthread_create(&th[t], NULL, res_worker, &J[t]);
  }
  res_worker(&J[0]);
  for (int t = 1; t < nthr; t++) pthread_join(th[t], NULL);
}

/* acc[g] <- (acc[g] + Ahi_g (2^14 Bhi_g^T) + 2^7 (Ahi_g Blo_g^T + Alo_g Bhi_g^T) + Alo_g Blo_g^T) mod m_g,
 * canonical residues in [0, m): rns.py:106-137 (and batched.py:96-127 with nb = 1).
 * lower_only: only entries with row >= column (the exact lower triangle). */
void or_accumulate(const int8_t* Ahi, const int8_t* Alo, const int8_t* Bhi, const int8_t* Blo, int G, i64 M, i64 N,
                   i64 KC, const int32_t* mods, int16_t* acc, int lower_only) {
  for (int g = 0; g < G; g++) {
    i64 m = mods[g];
    const int8_t *ah = Ahi + (i64)g * M * KC, *al = Alo + (i64)g * M * KC;
    const int8_t *bh = Bhi + (i64)g * N * KC, *bl = Blo + (i64)g * N * KC;
    for (i64 i = 0; i < M; i++)
      for (i64 j = 0; j < N; j++) {
        if (lower_only && j > i) continue;
        i64 s = 0;
        for (i64 k = 0; k < KC; k++) {
          i64 a = 128 * (i64)ah[i * KC + k] + al[i * KC + k];
          i64 b = 128 * (i64)bh[j * KC + k] + bl[j * KC + k];
          s += a * b;
        }
        int16_t* o = acc + ((i64)g * M + i) * N + j;
        i64 v = ((s % m) + m + *o) % m;
        *o = (int16_t)v;
      }
  }
}

/* CRT of residues acc (n, rows, N) int16 for the block rows x columns j0..j0+w: exact integers as W
 * two's-complement words per entry (entries e = i*w + jj, word-major output (W, rows*w)) plus the
 * bit length of v / ~v.  Same reconstruction as rns.py:227-238 with limbops.py:85-152:
 * y_i = acc_i * inv_i mod m_i (centred), k = round(sum y_i / m_i), X = sum y_i (M/m_i) - k M.
 * Mi: (n, W) words of M/m_i; Mw: (W) words of M. */
void or_crt_block(const int16_t* acc, i64 ldg, i64 N, i64 j0, i64 w, i64 rows, int n, const int32_t* mods,
                  const int32_t* inv, const u32* Mi, const u32* Mw, int W, int32_t* out, i64* bitlen) {
  i64 B = rows * w;
  i64* col = (i64*)malloc(sizeof(i64) * W);
  for (i64 e = 0; e < B; e++) {
    i64 i = e / w, jj = e % w;
    double ks = 0;
    for (int t = 0; t < W; t++) col[t] = 0;
    for (int g = 0; g < n; g++) {
      i64 m = mods[g];
      i64 a = acc[g * ldg + i * N + j0 + jj];
      i64 y = ((a * inv[g]) % m + m) % m;
      if (y > m / 2) y -= m;
      ks += (double)y / (double)m;
      for (int t = 0; t < W; t++) col[t] += y * (i64)Mi[(i64)g * W + t];
    }
    i64 k = (i64)floor(ks + 0.5);
    for (int t = 0; t < W; t++) col[t] -= k * (i64)Mw[t];
    i64 carry = 0;
    for (int t = 0; t < W; t++) {
      i64 v = col[t] + carry;
      out[(i64)t * B + e] = (int32_t)(u32)(v & (i64)MASK32);
      carry = v >> 32;
    }
  }
  free(col);
  or_bitlen(out, W, B, bitlen);
}

/* ---------------------------------------------------------------- Cholesky base case (wide fixed point)
 * Tiles are BT x BT entries of WL words, entry-major, F = 32*LF fraction bits: basecase.py:13-246. */

#define BC_MAXW 256

static int top_word(const u32* a, int WL) {
  for (int i = WL - 1; i > 0; i--)
    if (a[i]) return i;
  return 0;
}

/* r = (a*b) >> F truncated, computed on |a|, |b| from the column max(LF-2, la+lb) upwards only, where
 * t > 0 keeps the top t words of each operand; sign applied afterwards: basecase.py:31-53. */
void or_mulfx(u32* r, const u32* a, const u32* b, int t, int WL, int LF) {
  u32 x[BC_MAXW], y[BC_MAXW];
  memcpy(x, a, 4 * WL);
  memcpy(y, b, 4 * WL);
  int sa = x[WL - 1] >> 31, sb = y[WL - 1] >> 31;
  if (sa) neg_words(x, WL);
  if (sb) neg_words(y, WL);
  int ta = top_word(x, WL), tb = top_word(y, WL);
  int la = t ? (ta - t + 1 > 0 ? ta - t + 1 : 0) : 0;
  int lb = t ? (tb - t + 1 > 0 ? tb - t + 1 : 0) : 0;
  int kmin = (LF - 2 > la + lb) ? LF - 2 : la + lb;
  /* T = sum over i in [la,ta], j in [lb,tb], i+j >= kmin of x_i y_j 2^(32(i+j)), as 32-bit words
   * starting at word kmin (exact, 128-bit column sums). */
  int span = ta + tb + 3 - kmin;
  if (span < 1) span = 1;
  unsigned __int128 colsum[2 * BC_MAXW + 4];
  for (int c = 0; c < span; c++) colsum[c] = 0;
  for (int i = la; i <= ta; i++)
    for (int j = lb; j <= tb; j++)
      if (i + j >= kmin) colsum[i + j - kmin] += (unsigned __int128)((u64)x[i] * y[j]);
  memset(r, 0, 4 * WL);
  unsigned __int128 carry = 0;
  for (int c = 0; c < span; c++) {
    int k = kmin + c;
    unsigned __int128 v = colsum[c] + carry;
    if (k >= LF && k < LF + WL) r[k - LF] = (u32)v;
    carry = v >> 32;
  }
  if (sa ^ sb) neg_words(r, WL);
}

static void sub_words(u32* r, const u32* a, int WL) {
  i64 br = 0;
  for (int i = 0; i < WL; i++) {
    i64 t = (i64)r[i] - (i64)a[i] + br;
    r[i] = (u32)t;
    br = t >> 32;
  }
}

static void add_words(u32* r, const u32* a, int WL) {
  u64 c = 0;
  for (int i = 0; i < WL; i++) {
    u64 t = (u64)r[i] + a[i] + c;
    r[i] = (u32)t;
    c = t >> 32;
  }
}

/* Approximate double of a wide fixed-point value from its top three words: basecase.py:59-68. */
static double wide_to_double(const u32* a, int WL, int LF) {
  u32 x[BC_MAXW];
  memcpy(x, a, 4 * WL);
  int s = x[WL - 1] >> 31;
  if (s) neg_words(x, WL);
  int t = top_word(x, WL);
  double v = (double)x[t];
  if (t >= 1) v = v * 4294967296.0 + (double)x[t - 1];
  if (t >= 2) v = v * 4294967296.0 + (double)x[t - 2];
  v = ldexp(v, 32 * (t - 2 > 0 ? t - 2 : 0) - 32 * LF);
  return s ? -v : v;
}

/* Positive double -> wide fixed point (53 significant bits): basecase.py:69-78. */
static void wide_from_double(u32* r, double v, int WL, int LF) {
  memset(r, 0, 4 * WL);
  int e;
  double m = frexp(v, &e);
  u64 mi = (u64)ldexp(m, 53);
  int pos = e - 53 + 32 * LF;
  if (pos < 0) {
    mi >>= -pos;
    pos = 0;
  }
  int li = pos / 32, sh = pos % 32;
  unsigned __int128 w = ((unsigned __int128)mi) << sh;
  for (int k = 0; k < 4 && li + k < WL; k++) {
    r[li + k] = (u32)w;
    w >>= 32;
  }
}

/* r = d^(-1/2) by precision-doubling Newton steps r += r (1 - d r^2) / 2 from a double seed; the
 * warp-cooperative schedule of basecase.py:145-156 (full precision once t >= WL). */
void or_rsqrt(u32* r, const u32* d, int WL, int LF) {
  u32 t1[BC_MAXW], t2[BC_MAXW], one[BC_MAXW];
  wide_from_double(r, 1.0 / sqrt(wide_to_double(d, WL, LF)), WL, LF);
  memset(one, 0, 4 * WL);
  one[LF] = 1;
  for (int bits = 100;; bits *= 2) {
    int t = bits / 32 + 2;
    if (t >= WL) t = 0;
    or_mulfx(t1, r, r, t, WL, LF);
    or_mulfx(t2, t1, d, t, WL, LF);
    memcpy(t1, one, 4 * WL);
    sub_words(t1, t2, WL);
    or_mulfx(t2, r, t1, t, WL, LF);
    for (int i = 0; i < WL - 1; i++) t2[i] = (t2[i] >> 1) | (t2[i + 1] << 31);
    t2[WL - 1] = (u32)(((int32_t)t2[WL - 1]) >> 1);
    add_words(r, t2, WL);
    if (t == 0) break;
  }
}

/* In-place lower Cholesky of one BT x BT tile plus pivot reciprocals: basecase.py:158-193. */
void or_chol_tile(u32* T, u32* RI, int BT, int WL, int LF) {
  u32 v[BC_MAXW];
#define E(i, j) (T + ((size_t)(i) * BT + (j)) * WL)
  for (int k = 0; k < BT; k++) {
    u32 d[BC_MAXW];
    memcpy(d, E(k, k), 4 * WL);
    or_rsqrt(RI + (size_t)k * WL, d, WL, LF);
    or_mulfx(E(k, k), d, RI + (size_t)k * WL, 0, WL, LF);
    for (int i = k + 1; i < BT; i++) {
      or_mulfx(v, E(i, k), RI + (size_t)k * WL, 0, WL, LF);
      memcpy(E(i, k), v, 4 * WL);
    }
    for (int i = k + 1; i < BT; i++)
      for (int j = k + 1; j <= i; j++) {
        or_mulfx(v, E(i, k), E(j, k), 0, WL, LF);
        sub_words(E(i, j), v, WL);
      }
  }
#undef E
}

/* X = L^-1 of a lower tile, row by row, with the pivot reciprocals: basecase.py:195-226. */
void or_trinv_tile(const u32* Lt, const u32* RI, u32* X, int BT, int WL, int LF) {
  u32* S = (u32*)calloc((size_t)BT * BT * WL, 4);
  u32 acc[BC_MAXW], v[BC_MAXW];
  memset(X, 0, (size_t)BT * BT * WL * 4);
  for (int i = 0; i < BT; i++) {
    for (int j = 0; j < i; j++)
      for (int k = 0; k <= j; k++)
        or_mulfx(S + ((size_t)k * BT + j) * WL, Lt + ((size_t)i * BT + j) * WL, X + ((size_t)j * BT + k) * WL, 0,
                 WL, LF);
    for (int k = 0; k <= i; k++) {
      u32* xik = X + ((size_t)i * BT + k) * WL;
      if (k == i) {
        memcpy(xik, RI + (size_t)i * WL, 4 * WL);
        continue;
      }
      memset(acc, 0, 4 * WL);
      for (int j = k; j < i; j++) add_words(acc, S + ((size_t)k * BT + j) * WL, WL);
      or_mulfx(v, acc, RI + (size_t)i * WL, 0, WL, LF);
      neg_words(v, WL);
      memcpy(xik, v, 4 * WL);
    }
  }
  free(S);
}

/* Batched base case over nb tiles (AoS (nb, BT, BT, WL)); RINV (nb, BT, WL). */
void or_chol_tiles(u32* A, u32* RINV, i64 nb, int BT, int WL, int LF) {
  for (i64 b = 0; b < nb; b++)
    or_chol_tile(A + (size_t)b * BT * BT * WL, RINV + (size_t)b * BT * WL, BT, WL, LF);
}

void or_trinv_tiles(const u32* Lt, const u32* RINV, u32* X, i64 nb, int BT, int WL, int LF) {
  for (i64 b = 0; b < nb; b++)
    or_trinv_tile(Lt + (size_t)b * BT * BT * WL, RINV + (size_t)b * BT * WL, X + (size_t)b * BT * BT * WL, BT, WL,
                  LF);
}

/* basecase.py:228-245 (trsv_warp): solve L y = v for nvec vectors of BT entries with one factored tile
 * (upper part of Lt ignored): for j in order, y_j = v_j r_j, then v_i -= l_ij y_j for i > j.  V (nvec, BT,
 * WL) is overwritten by y. */
void or_trsv_tiles(const u32* Lt, const u32* RINV, u32* V, i64 nvec, int BT, int WL, int LF) {
  u32 p[256], t[256];
  for (i64 w = 0; w < nvec; w++) {
    u32* v = V + (size_t)w * BT * WL;
    for (int j = 0; j < BT; j++) {
      or_mulfx(p, v + (size_t)j * WL, RINV + (size_t)j * WL, 0, WL, LF);
      for (int k = 0; k < WL; k++) v[(size_t)j * WL + k] = p[k];
      for (int i = j + 1; i < BT; i++) {
        or_mulfx(t, Lt + ((size_t)i * BT + j) * WL, p, 0, WL, LF);
        sub_words(v + (size_t)i * WL, t, WL);
      }
    }
  }
}
