// CPU check of the Ozaki path's Chinese-remainder reconstruction (the same
// host/device code the reconstruction kernel runs): random integers X with
// |X| <= P/4 (the range the row scaling guarantees) are reduced modulo every
// modulus, reconstructed, and compared with X converted to double (within
// 1.5 units in the last place), with byte residues and with unreduced
// residues (r + a multiple of p, below 2^24), for a run-time and a fixed
// modulus count. Also checks the division-free reduction of int32 GEMM sums
// modulo each modulus (edges of the int32 range, around zero, random) and the
// CRT weights: W_t = 1 mod p_t and 0 mod p_s (s != t). Prints "OK <cases>" on
// success.
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../../spla_b200/csrc/kernels/ozaki_crt.cuh"

using namespace splab::oz;
typedef unsigned __int128 u128;
typedef __int128 i128;

static int mod_pos(i128 x, int p) {
  i128 r = x % p;
  if (r < 0) r += p;
  return int(r);
}

int main() {
  std::mt19937_64 rng(12345);
  long cases = 0;
  for (int n = 8; n <= 16; ++n) {
    const Crt c = make_crt(n);
    const u128 P = (u128(c.P_hi) << 64) | c.P_lo;
    for (int t = 0; t < n; ++t) {
      const u128 W = (u128(c.w_hi[t]) << 64) | c.w_lo[t];
      if (W >= P) { printf("FAIL weight >= P\n"); return 1; }
      for (int s = 0; s < n; ++s) {
        const int r = int(W % u128(c.p[s]));
        if (r != (s == t ? 1 : 0)) { printf("FAIL weight %d mod %d = %d\n", t, c.p[s], r); return 1; }
      }
    }
    const ReconParams rp = make_recon(c);
    const i128 quarter = i128(P / 4);
    for (int it = 0; it < 20000; ++it) {
      i128 X;
      const int kind = it % 6;
      if (kind == 0) X = quarter - i128(rng() % 1000);
      else if (kind == 1) X = -quarter + i128(rng() % 1000);
      else if (kind == 2) X = i128(int64_t(rng() % 2000001) - 1000000);
      else if (kind == 3) X = (i128(int64_t(rng())) * i128(rng() % 4096)) % (quarter + 1);
      else {
        u128 v = (u128(rng()) << 64) | rng();
        v %= u128(2 * quarter + 1);
        X = i128(v) - quarter;
      }
      int r[kMaxModuli];
      for (int t = 0; t < n; ++t) r[t] = mod_pos(X, c.p[t]);
      const long long hi = (long long)(X >> 64);
      const unsigned long long lo = (unsigned long long)X;
      const double want = (double)((long double)hi * 18446744073709551616.0L + (long double)lo);
      const double tol = (want < 0 ? -want : want) * 3.4e-16;  // 1.5 ulp
      auto bad = [&](double got) { return (got > want ? got - want : want - got) > tol; };
      const double got = crt_value<0, true>(r, rp);
      if (bad(got) || bad(crt_value<0, false>(r, rp))) {
        printf("FAIL n=%d it=%d got %.17g want %.17g\n", n, it, got, want);
        return 1;
      }
      if (n == 15 && bad(crt_value<15, true>(r, rp))) {
        printf("FAIL fixed n=15 it=%d\n", it);
        return 1;
      }
      if (n == 9 && bad(crt_value<9, true>(r, rp))) {
        printf("FAIL fixed n=9 it=%d\n", it);
        return 1;
      }
      // unreduced residues (sums of per-chunk residues, below 2^24)
      for (int t = 0; t < n; ++t)
        r[t] += c.p[t] * int(rng() % ((1u << 24) / unsigned(c.p[t]) - 1));
      const double got2 = crt_value<0, false>(r, rp);
      if (bad(got2)) {
        printf("FAIL unreduced n=%d it=%d got %.17g want %.17g\n", n, it, got2, want);
        return 1;
      }
      ++cases;
    }
  }
  // v mod p for int32 GEMM sums
  for (int t = 0; t < kMaxModuli; ++t) {
    const int p = kModuli[t];
    const ModMagic mm = make_mod_magic(p);
    auto check = [&](long long v) {
      long long want = v % p;
      if (want < 0) want += p;
      const int got = mod_residue(int(v), p, mm.c16, mm.off, mm.M);
      if (got != want) {
        printf("FAIL mod p=%d v=%lld got %d want %lld\n", p, v, got, want);
        return false;
      }
      return true;
    };
    for (long long v = -2147483648ll; v < -2147483648ll + 200000; ++v)
      if (!check(v)) return 1;
    for (long long v = 2147483647ll - 200000; v <= 2147483647ll; ++v)
      if (!check(v)) return 1;
    for (long long v = -300000; v <= 300000; ++v)
      if (!check(v)) return 1;
    for (int it = 0; it < 2000000; ++it)
      if (!check((long long)(int)(unsigned)rng())) return 1;
    cases += 1;
  }
  printf("OK %ld\n", cases);
  return 0;
}
