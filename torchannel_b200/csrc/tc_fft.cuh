// Hand-written mixed-radix (8, 4, 2, 3) complex FFTs on batches of rows held in
// shared memory.  Stockham autosort formulation (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC'08):
// every stage reads one buffer and writes the other in natural order, so no
// bit reversal pass is needed.  Twiddles come from a table
// tw[m] = exp(-2*pi*i*m/N), m < N, computed on the host in FP64 and staged in
// shared memory by the calling kernel.
//
// These transforms replace torch.fft.rfft2 / irfft2 of the reference
// (projection_fft.py:118,139; turbstats.py:165-173).
#pragma once
#include "tc_common.cuh"

namespace tc {

#define TC_FFT_MAX_STAGES 12

struct FftPlan {
  int n;
  int nstages;
  int radix[TC_FFT_MAX_STAGES];
};

// Host-side: factor n into stages of 8, 4, 2 and 3.  Returns 0 when n has any
// other prime factor.
inline int fft_make_plan(int n, FftPlan* p) {
  p->n = n;
  p->nstages = 0;
  if (n < 1) return 0;
  int m = n;
  while (m % 8 == 0) { if (p->nstages >= TC_FFT_MAX_STAGES) return 0; p->radix[p->nstages++] = 8; m /= 8; }
  while (m % 4 == 0) { if (p->nstages >= TC_FFT_MAX_STAGES) return 0; p->radix[p->nstages++] = 4; m /= 4; }
  while (m % 2 == 0) { if (p->nstages >= TC_FFT_MAX_STAGES) return 0; p->radix[p->nstages++] = 2; m /= 2; }
  while (m % 3 == 0) { if (p->nstages >= TC_FFT_MAX_STAGES) return 0; p->radix[p->nstages++] = 3; m /= 3; }
  return m == 1;
}

// Multiply by -i (forward) or +i (inverse).
template <class T, bool INV> __device__ __forceinline__ cpx<T> mul_mi(cpx<T> a) {
  return INV ? cmake<T>(-a.y, a.x) : cmake<T>(a.y, -a.x);
}

template <class T, bool INV> __device__ __forceinline__ void dft2(cpx<T>* v) {
  cpx<T> a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <class T, bool INV> __device__ __forceinline__ void dft4(cpx<T>* v) {
  cpx<T> s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
  cpx<T> s13 = cadd(v[1], v[3]), d13 = mul_mi<T, INV>(csub(v[1], v[3]));
  v[0] = cadd(s02, s13);
  v[2] = csub(s02, s13);
  v[1] = cadd(d02, d13);
  v[3] = csub(d02, d13);
}

// radix 8 from two radix-4 halves: y_k = E_k + W8^k O_k, y_{k+4} = E_k - W8^k O_k
template <class T, bool INV> __device__ __forceinline__ void dft8(cpx<T>* v) {
  const T r = (T)0.70710678118654752440084436210485;  // 1/sqrt(2)
  cpx<T> e[4] = {v[0], v[2], v[4], v[6]};
  cpx<T> o[4] = {v[1], v[3], v[5], v[7]};
  dft4<T, INV>(e);
  dft4<T, INV>(o);
  {  // W8^1 = (1 -/+ i)/sqrt(2)
    T a = o[1].x, b = o[1].y;
    o[1] = INV ? cmake<T>((a - b) * r, (a + b) * r) : cmake<T>((a + b) * r, (b - a) * r);
  }
  o[2] = mul_mi<T, INV>(o[2]);  // W8^2 = -/+ i
  {  // W8^3 = (-1 -/+ i)/sqrt(2)
    T a = o[3].x, b = o[3].y;
    o[3] = INV ? cmake<T>((-a - b) * r, (a - b) * r) : cmake<T>((b - a) * r, -(a + b) * r);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    v[q] = cadd(e[q], o[q]);
    v[q + 4] = csub(e[q], o[q]);
  }
}

// y1 = x0 - (x1+x2)/2 -/+ i s (x1-x2), y2 = x0 - (x1+x2)/2 +/- i s (x1-x2), s = sqrt(3)/2
template <class T, bool INV> __device__ __forceinline__ void dft3(cpx<T>* v) {
  const T s = (T)0.86602540378443864676372317075294;
  cpx<T> x0 = v[0], sum = cadd(v[1], v[2]), dif = csub(v[1], v[2]);
  cpx<T> t = cmake<T>(x0.x - (T)0.5 * sum.x, x0.y - (T)0.5 * sum.y);
  cpx<T> r = mul_mi<T, INV>(cscale(dif, s));
  v[0] = cadd(x0, sum);
  v[1] = cadd(t, r);
  v[2] = csub(t, r);
}

// Shared-memory layout of the transform buffers: element e of a row sits at
// padi(e) = e + e/8 (FP64 complex) or e + e/16 (FP32 complex).  The early
// Stockham stages store at a stride of R elements, which without the pad
// would put a whole warp on one bank group.
template <class T> __host__ __device__ __forceinline__ constexpr int pad_shift() {
  return sizeof(cpx<T>) >= 16 ? 3 : 4;
}
template <class T> __device__ __forceinline__ int padi(int e) { return e + (e >> pad_shift<T>()); }
// Row pitch of a padded row of n elements.
template <class T> __host__ __device__ __forceinline__ int padded_len(int n) {
  return n + (n >> pad_shift<T>()) + 1;
}

// One Stockham stage over `batch` rows (row pitch `rs`, padded layout).  NC
// and NSC are the transform length and current span when known at compile
// time (0: use the run-time n and Ns).
template <class T, bool INV, int R, int NC, int NSC>
__device__ __forceinline__ void fft_stage(const cpx<T>* __restrict__ x, cpx<T>* __restrict__ y, int batch,
                                          int rs, int n_rt, int Ns_rt, const cpx<T>* __restrict__ tw, int tid,
                                          int nthr) {
  const int n = NC ? NC : n_rt;
  const int Ns = NC ? NSC : Ns_rt;
  const int nr = n / R;
  const int fac = n / (Ns * R);
  const int total = batch * nr;
  for (int idx = tid; idx < total; idx += nthr) {
    const int b = idx / nr;
    const int j = idx - b * nr;
    const cpx<T>* xb = x + (size_t)b * rs;
    cpx<T>* yb = y + (size_t)b * rs;
    const int k = j % Ns;
    cpx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = xb[padi<T>(j + r * nr)];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        cpx<T> w = tw[r * k * fac];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    if (R == 2) dft2<T, INV>(v);
    else if (R == 4) dft4<T, INV>(v);
    else if (R == 8) dft8<T, INV>(v);
    else dft3<T, INV>(v);
    const int o = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) yb[padi<T>(o + r * Ns)] = v[r];
  }
}

// Stage a twiddle table of n entries into shared memory (callers then pass
// the shared copy to fft_rows).  No trailing barrier: fft_rows callers
// synchronise after loading their data.
template <class T>
__device__ __forceinline__ void stage_twiddles(cpx<T>* dst, const cpx<T>* __restrict__ src, int n, int tid, int nthr) {
  for (int e = tid; e < n; e += nthr) dst[e] = src[e];
}

// Radix of the stage that starts at span NS of a length-N transform.
template <int N, int NS> struct NextRadix {
  static constexpr int rem = N / NS;
  static constexpr int value = (rem % 8 == 0) ? 8 : (rem % 4 == 0) ? 4 : (rem % 2 == 0) ? 2 : 3;
};

// Compile-time-length batched FFT: returns the index (0: a, 1: b) of the
// buffer holding the result.
template <class T, bool INV, int N, int NS>
__device__ __forceinline__ int fft_rows_c(cpx<T>* a, cpx<T>* b, int batch, int rs, const cpx<T>* __restrict__ tw,
                                          int tid, int nthr) {
  if constexpr (NS >= N) {
    return 0;
  } else {
    constexpr int R = NextRadix<N, NS>::value;
    fft_stage<T, INV, R, N, NS>(a, b, batch, rs, N, NS, tw, tid, nthr);
    __syncthreads();
    return 1 ^ fft_rows_c<T, INV, N, NS * R>(b, a, batch, rs, tw, tid, nthr);
  }
}

// Batched in-smem FFT (padded layout).  Data starts in buf0; returns the
// index (0/1) of the buffer that holds the result.  Unnormalised in both
// directions.  All threads of the block must call it; it synchronises.
// Common lengths use compile-time plans; others the run-time plan.
template <class T, bool INV>
__device__ int fft_rows(cpx<T>* buf0, cpx<T>* buf1, int batch, int rs, const FftPlan& pl,
                        const cpx<T>* __restrict__ tw, int tid, int nthr) {
  switch (pl.n) {
    case 64: return fft_rows_c<T, INV, 64, 1>(buf0, buf1, batch, rs, tw, tid, nthr);
    case 96: return fft_rows_c<T, INV, 96, 1>(buf0, buf1, batch, rs, tw, tid, nthr);
    case 128: return fft_rows_c<T, INV, 128, 1>(buf0, buf1, batch, rs, tw, tid, nthr);
    case 192: return fft_rows_c<T, INV, 192, 1>(buf0, buf1, batch, rs, tw, tid, nthr);
    case 256: return fft_rows_c<T, INV, 256, 1>(buf0, buf1, batch, rs, tw, tid, nthr);
    case 384: return fft_rows_c<T, INV, 384, 1>(buf0, buf1, batch, rs, tw, tid, nthr);
    case 768: return fft_rows_c<T, INV, 768, 1>(buf0, buf1, batch, rs, tw, tid, nthr);
    default: break;
  }
  cpx<T>* bufs[2] = {buf0, buf1};
  int cur = 0;
  int Ns = 1;
  for (int s = 0; s < pl.nstages; ++s) {
    int R = pl.radix[s];
    if (R == 8) fft_stage<T, INV, 8, 0, 0>(bufs[cur], bufs[cur ^ 1], batch, rs, pl.n, Ns, tw, tid, nthr);
    else if (R == 4) fft_stage<T, INV, 4, 0, 0>(bufs[cur], bufs[cur ^ 1], batch, rs, pl.n, Ns, tw, tid, nthr);
    else if (R == 2) fft_stage<T, INV, 2, 0, 0>(bufs[cur], bufs[cur ^ 1], batch, rs, pl.n, Ns, tw, tid, nthr);
    else fft_stage<T, INV, 3, 0, 0>(bufs[cur], bufs[cur ^ 1], batch, rs, pl.n, Ns, tw, tid, nthr);
    Ns *= R;
    cur ^= 1;
    __syncthreads();
  }
  return cur;
}

}  // namespace tc
