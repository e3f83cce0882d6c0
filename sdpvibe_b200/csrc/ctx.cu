// RNS context: moduli, decomposition tables and CRT tables for one limb count, built on the host
// with a small unsigned bignum and uploaded once per (limb count, device).
// The moduli rule and table definitions follow sdpvibe/rns.py:22-35 and 166-191.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

struct Big {  // little-endian 32-bit words
  std::vector<u32> w;
  void mul_small(u32 m) {
    u64 c = 0;
    for (auto& x : w) {
      u64 t = (u64)x * m + c;
      x = (u32)t;
      c = t >> 32;
    }
    if (c) w.push_back((u32)c);
  }
  u32 divmod_small(u32 m) {  // in place quotient, returns remainder
    u64 r = 0;
    for (size_t i = w.size(); i-- > 0;) {
      u64 cur = (r << 32) | w[i];
      w[i] = (u32)(cur / m);
      r = cur % m;
    }
    while (!w.empty() && w.back() == 0) w.pop_back();
    return (u32)r;
  }
  u32 mod_small(u32 m) const {
    u64 r = 0;
    for (size_t i = w.size(); i-- > 0;) r = ((r << 32) | w[i]) % m;
    return (u32)r;
  }
  int bitlen() const {
    for (size_t i = w.size(); i-- > 0;)
      if (w[i]) return 32 * (int)i + 32 - __builtin_clz(w[i]);
    return 0;
  }
  // Signed base-256 digits in [-128, 128), `count` of them (x must fit).
  std::vector<int> sdigits256(int count) const {
    std::vector<int> out(count);
    int carry = 0;
    for (int t = 0; t < count; t++) {
      int b = (t / 4 < (int)w.size()) ? (int)((w[t / 4] >> (8 * (t % 4))) & 255u) : 0;
      int v = b + carry;
      int r = ((v + 128) & 255) - 128;
      out[t] = r;
      carry = (v - r) / 256;
    }
    return out;
  }
};

std::vector<int> primes_desc(int hi, int lo) {  // primes p with lo < p <= hi, descending
  std::vector<char> s(hi + 1, 1);
  s[0] = s[1] = 0;
  for (int p = 2; (long)p * p <= hi; p++)
    if (s[p])
      for (int q = p * p; q <= hi; q += p) s[q] = 0;
  std::vector<int> out;
  for (int p = hi; p > lo; p--)
    if (s[p]) out.push_back(p);
  return out;
}

long powmod(long b, long e, long m) {
  long r = 1 % m;
  b %= m;
  while (e > 0) {
    if (e & 1) r = r * b % m;
    b = b * b % m;
    e >>= 1;
  }
  return r;
}

long invmod(long a, long m) {  // a^-1 mod m (m prime)
  return powmod(((a % m) + m) % m, m - 2, m);
}

template <class T>
int upload(T** dst, const std::vector<T>& v) {
  if (cudaMalloc((void**)dst, sizeof(T) * std::max<size_t>(v.size(), 1)) != cudaSuccess) return SDPV_ENOMEM;
  if (!v.empty() && cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return SDPV_ECUDA;
  return SDPV_OK;
}

}  // namespace

extern "C" int sdpv_ctx_create(int L, sdpv_ctx** out) { return sdpv_ctx_create_g(L, 16, out); }

// G: the moduli count is the least multiple of G that meets the bound (the reference uses G = 16); any G
// gives the same exact products, a smaller one fewer moduli
extern "C" int sdpv_ctx_create_g(int L, int G, sdpv_ctx** out) {
  if (!out || L < 1 || L > 160 || G < 1 || G > 16 || (G & (G - 1))) return SDPV_EINVAL;
  // moduli: rns.py:168-173; M > 4 * 2^17 * 2^(2(32L-1)) <=> bitlen(M) >= 64L + 18
  std::vector<int> mods;
  Big M;
  M.w = {1};
  for (int p : primes_desc(32639, 1 << 14)) {
    if (M.bitlen() >= 64 * L + 18 && mods.size() % G == 0) break;
    mods.push_back(p);
    M.mul_small((u32)p);
  }
  int n = (int)mods.size();
  if (M.bitlen() < 64 * L + 18) return SDPV_EINVAL;  // not enough primes below 2^15
  int E = ((M.bitlen() + 7) / 8 + 2 + 7) / 8 * 8;     // rns.py:186
  int NB = 4 * L;

  sdpv_ctx* c = new sdpv_ctx();
  sdpv::CtxDev& d = c->d;
  cudaGetDevice(&c->device);
  d.L = L;
  d.n = n;
  d.E = E;
  d.W = E / 4;
  d.npad = (n + 127) / 128 * 128;
  d.kt = (NB + 2 + 127) / 128;   // limb bytes + a constant byte + a sign byte
  d.ktc = (n + 127) / 128;
  d.npad16 = (n + 31) / 32 * 32;
  d.Epad = (E + 127) / 128 * 128;

  std::vector<int32_t> vm(n), vc14(n), vc1(n), vc1m2(n), vinv(n);
  std::vector<float> vminv(n);
  int ngroups = d.npad / 128;
  std::vector<uint8_t> tab((size_t)ngroups * 2 * d.kt * 128 * 128, 0);
  std::vector<uint8_t> tabu(tab.size(), 0);
  auto put_u = [&](int grp, int row, int j, long t) {   // canonical t in [0, m) as unsigned digits
    int kt = j / 128, col = j % 128;
    u32 off = sw128_off(row, col / 16) + (col % 16);
    tabu[(((size_t)grp * 2 + 0) * d.kt + kt) * 128 * 128 + off] = (uint8_t)(t & 127);
    tabu[(((size_t)grp * 2 + 1) * d.kt + kt) * 128 * 128 + off] = (uint8_t)(t >> 7);
  };
  for (int g = 0; g < n; g++) {
    long m = mods[g];
    vm[g] = (int32_t)m;
    vminv[g] = (float)(1.0 / (double)m);
    vc14[g] = (int32_t)powmod(2, 14, m);
    long tsum = 0;
    int grp = g / 128, row = g % 128;
    for (int j = 0; j < NB; j++) {
      long t = powmod(256, j, m);
      put_u(grp, row, j, t);
      if (t > m / 2) t -= m;  // centred
      tsum += t;
      long lo = ((t + 64) % 128 + 128) % 128 - 64;
      long hi = (t - lo) / 128;
      int kt = j / 128, col = j % 128;
      size_t base_lo = (((size_t)grp * 2 + 0) * d.kt + kt) * 128 * 128;
      size_t base_hi = (((size_t)grp * 2 + 1) * d.kt + kt) * 128 * 128;
      u32 off = sw128_off(row, col / 16) + (col % 16);
      tab[base_lo + off] = (uint8_t)(int8_t)lo;
      tab[base_hi + off] = (uint8_t)(int8_t)hi;
    }
    long c1 = ((128 * tsum) % m + m) % m;
    long c2 = powmod(2, 32L * L, m);
    put_u(grp, row, NB, (m - c2) % m);        // unsigned table: the sign byte subtracts 2^(32L)
    vc1[g] = (int32_t)c1;
    vc1m2[g] = (int32_t)(c1 - c2);
    // Column NB multiplies a constant byte 1 (adds C1), column NB+1 the sign byte (subtracts C2):
    // the tensor-core product then is congruent to the entry itself.
    long extra[2] = {c1 > m / 2 ? c1 - m : c1, (c2 == 0) ? 0 : ((m - c2) > m / 2 ? (m - c2) - m : (m - c2))};
    for (int x = 0; x < 2; x++) {
      long t = extra[x];
      long lo = ((t + 64) % 128 + 128) % 128 - 64;
      long hi = (t - lo) / 128;
      int j = NB + x, kt = j / 128, col = j % 128;
      u32 off = sw128_off(row, col / 16) + (col % 16);
      tab[(((size_t)grp * 2 + 0) * d.kt + kt) * 128 * 128 + off] = (uint8_t)(int8_t)lo;
      tab[(((size_t)grp * 2 + 1) * d.kt + kt) * 128 * 128 + off] = (uint8_t)(int8_t)hi;
    }
    Big Mi = M;
    Mi.divmod_small((u32)m);
    vinv[g] = (int32_t)invmod(Mi.mod_small((u32)m), m);
  }
  // CRT digits: Ct[t][i] = signed base-256 digit t of M/m_i; B operand rows = digits, K = moduli.
  int nchunks = d.Epad / 128;
  std::vector<uint8_t> ct((size_t)nchunks * d.ktc * 128 * 128, 0);
  for (int i = 0; i < n; i++) {
    Big Mi = M;
    Mi.divmod_small((u32)mods[i]);
    std::vector<int> dg = Mi.sdigits256(E);
    for (int t = 0; t < E; t++) {
      int chunk = t / 128, row = t % 128, kt = i / 128, col = i % 128;
      size_t base = ((size_t)chunk * d.ktc + kt) * 128 * 128;
      ct[base + sw128_off(row, col / 16) + (col % 16)] = (uint8_t)(int8_t)dg[t];
    }
  }
  std::vector<int> mdg = M.sdigits256(E);
  std::vector<int32_t> vmd(d.Epad, 0);
  for (int t = 0; t < E; t++) vmd[t] = mdg[t];

  int st = SDPV_OK;
  if (!st) st = upload(&d.mods, vm);
  if (!st) st = upload(&d.minv, vminv);
  if (!st) st = upload(&d.c14, vc14);
  if (!st) st = upload(&d.c1, vc1);
  if (!st) st = upload(&d.c1m2, vc1m2);
  if (!st) st = upload(&d.inv, vinv);
  if (!st) st = upload(&d.md, vmd);
  if (!st) st = upload(&d.tab, tab);
  if (!st) st = upload(&d.tabu, tabu);
  if (!st) st = upload(&d.ct, ct);
  c->mods_host = new int32_t[n];
  memcpy(c->mods_host, vm.data(), sizeof(int32_t) * n);
  if (st) {
    sdpv_ctx_destroy(c);
    return st;
  }
  *out = c;
  return SDPV_OK;
}

extern "C" int sdpv_ctx_destroy(sdpv_ctx* c) {
  if (!c) return SDPV_OK;
  sdpv::CtxDev& d = c->d;
  void* ptrs[] = {d.mods, d.minv, d.c14, d.c1, d.c1m2, d.inv, d.md, d.tab, d.tabu, d.ct};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete[] c->mods_host;
  delete c;
  return SDPV_OK;
}

extern "C" int sdpv_ctx_query(const sdpv_ctx* c, int* n, int* E, int* W) {
  if (!c) return SDPV_EINVAL;
  if (n) *n = c->d.n;
  if (E) *E = c->d.E;
  if (W) *W = c->d.W;
  return SDPV_OK;
}

extern "C" int sdpv_ctx_moduli(const sdpv_ctx* c, int32_t* mods_host) {
  if (!c || !mods_host) return SDPV_EINVAL;
  memcpy(mods_host, c->mods_host, sizeof(int32_t) * c->d.n);
  return SDPV_OK;
}

extern "C" int sdpv_version(void) { return 1; }
