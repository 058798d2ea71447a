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
#include <cmath>
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
      // unreduced residues (combinations of per-chunk residue sums, below 2^26)
      for (int t = 0; t < n; ++t)
        r[t] += c.p[t] * int(rng() % ((1u << 26) / unsigned(c.p[t]) - 1));
      const double got2 = crt_value<0, false>(r, rp);
      if (bad(got2)) {
        printf("FAIL unreduced n=%d it=%d got %.17g want %.17g\n", n, it, got2, want);
        return 1;
      }
      ++cases;
    }
    // complex products from three real ones: random P0, P1 (|Re| < 2^57), Im
    // with |Im| <= P/4 and P2 chosen to match; residues combined per modulus
    // (byte residues, or unreduced int32 sums with the off24 offsets)
    for (int it = 0; it < 4000; ++it) {
      const int conj = it & 1;
      const i128 im = (i128(int64_t(rng())) * i128(rng() % 64)) % (quarter + 1);
      const i128 P0 = i128(int64_t(rng() >> 8)), P1 = i128(int64_t(rng() >> 8));
      // conj: Re = P0 + P1, Im = P2 - P0 + P1; else Re = P0 - P1, Im = P2 - P0 - P1
      const i128 P2 = conj ? im + P0 - P1 : im + P0 + P1;
      const i128 re_x = conj ? P0 + P1 : P0 - P1;
      int rr[kMaxModuli], ri[kMaxModuli];
      for (int t = 0; t < n; ++t) {
        const int pt = c.p[t];
        const bool bytes = (it >> 1) & 1;
        const int off = bytes ? pt : rp.off24[t];
        // byte residues, or unreduced sums below 2^24
        const int extra = bytes ? 0 : pt * int(rng() % ((1u << 24) / unsigned(pt) - 1));
        combine3(mod_pos(P0, pt) + (bytes ? 0 : extra), mod_pos(P1, pt), mod_pos(P2, pt), off, conj,
                 rr[t], ri[t]);
      }
      const double want_im = double((long double)im);
      const double g_re = crt_value<0, false>(rr, rp), g_im = crt_value<0, false>(ri, rp);
      const double w_re = double((long double)re_x);
      if (std::fabs(g_re - w_re) > std::fabs(w_re) * 3.4e-16 ||
          std::fabs(g_im - want_im) > std::fabs(want_im) * 3.4e-16) {
        printf("FAIL combine n=%d it=%d re %.17g/%.17g im %.17g/%.17g\n", n, it, g_re, w_re,
               g_im, want_im);
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
