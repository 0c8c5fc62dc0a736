// Register-resident complex FFTs of rows of length N = N1 * 16, one or two
// rows per warp, FP64.  Cooley-Tukey with one transpose (the "four-step"
// split N = N1 N2, N2 = 16):
//   pass 1: lane n2 of a row loads x[N2 n1 + n2] (n1 < N1), does an N1-point
//           DFT in registers and multiplies term k1 by W_N^(n2 k1);
//   exchange through a padded per-row shared tile (warp-synchronous);
//   pass 2: lane k1 loads the N2 terms of column k1, does an N2-point DFT and
//           owns X[k1 + N1 k2] (k2 < N2).
// Loads of pass 1 and stores of pass 2 are coalesced runs of N2 / N1
// elements; no block barrier is taken.  The small DFTs are built at compile
// time from radix 2, 3, 4 and 8 blocks with constant twiddles, which are
// computed here from their Taylor series (no run-time trigonometry).
// Unnormalised in both directions, like fft_rows.
#pragma once
#include <type_traits>

#include "tc_common.cuh"
#include "tc_fft.cuh"

namespace tc {

// ---- compile-time twiddles ------------------------------------------------
// sin and cos on [0, pi/4] from their Taylor series (terms to x^29; the
// remainder is below 1e-30 there).
constexpr double cx_sin_series(double x) {
  double term = x, sum = x;
  for (int k = 1; k < 15; ++k) {
    term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double cx_cos_series(double x) {
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 15; ++k) {
    term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
    sum += term;
  }
  return sum;
}
// cos and sin of 2 pi e / n, reduced to a quadrant and then to [0, pi/4].
struct CxCS { double c, s; };
constexpr CxCS cx_cossin(int e, int n) {
  const double half_pi = 1.5707963267948966;
  const int ee = ((e % n) + n) % n;
  const int q = (4 * ee) / n;               // quadrant
  const int r = 4 * ee - q * n;             // angle within it: (r / n) * pi/2
  double c = 0.0, s = 0.0;
  if (2 * r <= n) {
    const double a = (double)r / (double)n * half_pi;
    c = cx_cos_series(a); s = cx_sin_series(a);
  } else {
    const double b = (double)(n - r) / (double)n * half_pi;
    c = cx_sin_series(b); s = cx_cos_series(b);
  }
  switch (q) {
    case 0: return CxCS{c, s};
    case 1: return CxCS{-s, c};
    case 2: return CxCS{-c, -s};
    default: return CxCS{s, -c};
  }
}

// a * W_N^E with W_N = exp(-2 pi i / N) (forward) or its conjugate (inverse);
// exact for the multiples of a quarter turn.  T = double or float (the
// constants are rounded once to T).
template <int E, int N, bool INV, class T = double> __device__ __forceinline__ cpx<T> twc(cpx<T> a) {
  constexpr int e = ((E % N) + N) % N;
  if constexpr (e == 0) {
    return a;
  } else if constexpr (4 * e == N) {
    return mul_mi<T, INV>(a);
  } else if constexpr (2 * e == N) {
    return cmake<T>(-a.x, -a.y);
  } else if constexpr (4 * e == 3 * N) {
    return mul_mi<T, !INV>(a);
  } else {
    constexpr CxCS w = cx_cossin(e, N);
    constexpr T c = (T)w.c, s = (T)w.s;
    return INV ? cmake<T>(a.x * c - a.y * s, a.x * s + a.y * c)
               : cmake<T>(a.x * c + a.y * s, a.y * c - a.x * s);
  }
}

template <int B, int E, class F> __device__ __forceinline__ void static_for(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

// ---- small DFTs in registers (natural order in and out) -------------------
template <int N, bool INV, class T = double> struct Dft;
template <bool INV, class T> struct Dft<1, INV, T> { static __device__ __forceinline__ void run(cpx<T>*) {} };
template <bool INV, class T> struct Dft<2, INV, T> {
  static __device__ __forceinline__ void run(cpx<T>* v) { dft2<T, INV>(v); }
};
template <bool INV, class T> struct Dft<3, INV, T> {
  static __device__ __forceinline__ void run(cpx<T>* v) { dft3<T, INV>(v); }
};
template <bool INV, class T> struct Dft<4, INV, T> {
  static __device__ __forceinline__ void run(cpx<T>* v) { dft4<T, INV>(v); }
};
template <bool INV, class T> struct Dft<8, INV, T> {
  static __device__ __forceinline__ void run(cpx<T>* v) { dft8<T, INV>(v); }
};
// N = R M: R-point DFTs of the stride-M subsets, twiddles W_N^(n2 k1), then
// M-point DFTs; output index k1 + R k2.
template <int N> constexpr int dft_first_radix() {
  return (N % 8 == 0 && N > 8) ? 8 : (N % 4 == 0) ? 4 : (N % 3 == 0) ? 3 : 2;
}
template <int N, bool INV, class T> struct Dft {
  static __device__ __forceinline__ void run(cpx<T>* v) {
    constexpr int R = dft_first_radix<N>();
    constexpr int M = N / R;
    static_assert(R * M == N, "unsupported DFT length");
    cpx<T> t[N];
    static_for<0, M>([&](auto I2) {
      constexpr int n2 = decltype(I2)::value;
      cpx<T> a[R];
#pragma unroll
      for (int n1 = 0; n1 < R; ++n1) a[n1] = v[M * n1 + n2];
      Dft<R, INV, T>::run(a);
      static_for<0, R>([&](auto K1) {
        constexpr int k1 = decltype(K1)::value;
        t[k1 * M + n2] = twc<n2 * k1, N, INV, T>(a[k1]);
      });
    });
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
      cpx<T> b[M];
#pragma unroll
      for (int n2 = 0; n2 < M; ++n2) b[n2] = t[k1 * M + n2];
      Dft<M, INV, T>::run(b);
#pragma unroll
      for (int k2 = 0; k2 < M; ++k2) v[k1 + R * k2] = b[k2];
    }
  }
};

// ---- row transform of length N = 16 K -----------------------------------
// Split N = N1 N2 with N1 = K, N2 = 16 for K <= 32, and N1 = K / 2, N2 = 32
// above (N = 576, 768, 1024), so that a row's lanes, max(N1, N2), fit in a
// warp.
template <int K> struct RowFft {
  static constexpr int N1 = K <= 32 ? K : K / 2;
  static constexpr int N2 = K <= 32 ? 16 : 32;
  static constexpr int N = N1 * N2;
  static constexpr int LANES = N1 > N2 ? N1 : N2;         // lanes a row needs
  static constexpr int RPW = 32 / LANES;                  // rows per warp
  static constexpr int TP = N2 + 1;                       // tile pitch (complex)
  static constexpr int TILE = N1 * TP;                    // tile size per row (complex)
  static_assert(N == 16 * K && LANES <= 32, "unsupported row length");
};

// Pass 1 for lane n2: v[n1] = x[N2 n1 + n2] -> DFT_N1 -> times W_N^(n2 k1),
// stored to tile[k1 * TP + n2].  `ld(e)` returns element e of the row.
template <int K, bool INV, class LD>
__device__ __forceinline__ void rowfft_pass1(LD ld, int n2, cpx<double>* tile, const cpx<double>* __restrict__ tw) {
  using RF = RowFft<K>;
  cpx<double> v[RF::N1];
#pragma unroll
  for (int n1 = 0; n1 < RF::N1; ++n1) v[n1] = ld(RF::N2 * n1 + n2);
  Dft<RF::N1, INV>::run(v);
#pragma unroll
  for (int k1 = 0; k1 < RF::N1; ++k1) {
    cpx<double> w = tw[n2 * k1];
    if (INV) w.y = -w.y;
    tile[k1 * RF::TP + n2] = k1 == 0 ? v[0] : cmul(v[k1], w);
  }
}

// Pass 1 on values already in registers: v[n1] = x[N2 n1 + n2].
template <int K, bool INV>
__device__ __forceinline__ void rowfft_pass1_regs(cpx<double> (&v)[RowFft<K>::N1], int n2, cpx<double>* tile,
                                                  const cpx<double>* __restrict__ tw) {
  using RF = RowFft<K>;
  Dft<RF::N1, INV>::run(v);
#pragma unroll
  for (int k1 = 0; k1 < RF::N1; ++k1) {
    cpx<double> w = tw[n2 * k1];
    if (INV) w.y = -w.y;
    tile[k1 * RF::TP + n2] = k1 == 0 ? v[0] : cmul(v[k1], w);
  }
}

// Pass 2 for lane k1: b[n2] = tile[k1 * TP + n2] -> DFT_N2; `st(e, val)`
// receives element e = k1 + N1 k2 of the transformed row.
template <int K, bool INV, class ST>
__device__ __forceinline__ void rowfft_pass2(ST st, int k1, const cpx<double>* tile) {
  using RF = RowFft<K>;
  cpx<double> b[RF::N2];
#pragma unroll
  for (int n2 = 0; n2 < RF::N2; ++n2) b[n2] = tile[k1 * RF::TP + n2];
  Dft<RF::N2, INV>::run(b);
#pragma unroll
  for (int k2 = 0; k2 < RF::N2; ++k2) st(k1 + RF::N1 * k2, b[k2]);
}

// Lengths with a register transform: K = N / 16 in {4, 6, 8, 9, 12, 16, 18,
// 24, 32, 36, 48, 64} (N = 64 .. 1024).
__host__ __device__ inline bool rowfft_supported(int n) {
  if (n % 16) return false;
  switch (n / 16) {
    case 4: case 6: case 8: case 9: case 12: case 16: case 18: case 24: case 32: case 36: case 48: case 64:
      return true;
    default:
      return false;
  }
}

}  // namespace tc
