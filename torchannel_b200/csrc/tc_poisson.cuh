// Kernel (c): pressure Poisson solve  L p = div(u**)/dt  with periodic x/y and
// Neumann walls (projection_fft.py:3-165), as
//   [divergence + real FFT along x] -> [FFT along y] -> [Thomas along z per
//   (kx, ky), coefficients built on the fly] -> [inverse FFT along y] ->
//   [inverse real FFT along x -> p].
// Spectral intermediate X[kx][k][j] (complex, kx < nx/2+1): the x transform
// writes it transposed so that every later pass reads contiguous rows/columns.
// Two real rows travel as one complex row through the x transforms
// (z = a + i b; A = (Z + conj Z(-m))/2, B = (Z - conj Z(-m))/(2i)).
#pragma once
#include <cooperative_groups.h>

#include "tc_common.cuh"
#include "tc_fft.cuh"
#include "tc_fft_reg.cuh"
#undef TC_FILE_ID
#define TC_FILE_ID 3

namespace tc {

struct PoissonTabs {
  const double* k2x;  // nx/2+1: modified wavenumber squared (projection_fft.py:26-39)
  const double* k2y;  // ny
  const double* cl;   // nz: 1/(dz_c[k] dz_f[k])          (projection_fft.py:48)
  const double* cr;   // nz: 1/(dz_c[k+1] dz_f[k])        (projection_fft.py:49)
};

// Divergence (utils.py:226-240) of (u, v, w) scaled by `scale`, or a given
// FP64 cell field times `scale` when u == nullptr; then forward real FFT along
// x of JT rows of plane k.  Writes X[m][k][j] for m < nx/2+1.  The spectrum
// and the transforms are FP64 whatever the velocity storage type: pressure
// errors reach the post-projection divergence amplified by dt/(dz_c dz_f),
// which is ~1e4 next to the walls of a stretched grid.
template <class T>
__global__ void __launch_bounds__(256) k_div_fftx(Grid<T> g, const T* __restrict__ u, const T* __restrict__ v,
                                                  const T* __restrict__ w, const double* __restrict__ field,
                                                  cpx<double>* __restrict__ X, FftPlan plx,
                                                  const cpx<double>* __restrict__ twx, double scale, int JT) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxh = nx / 2 + 1;
  const int rs = padded_len<double>(nx);
  cpx<double>* b0 = reinterpret_cast<cpx<double>*>(smraw);
  cpx<double>* b1 = b0 + (JT / 2) * rs;
  cpx<double>* stw = b1 + (JT / 2) * rs;  // twiddles (nx)
  const int k = blockIdx.y, j0 = blockIdx.x * JT;
  const int tid = threadIdx.x, nthr = blockDim.x;
  stage_twiddles(stw, twx, nx, tid, nthr);
  // grid reciprocals are read only on the divergence path (a field-only
  // caller may pass a grid without z tables)
  const double idx = (double)g.idx, idy = (double)g.idy;
  const double idzf = (u != nullptr) ? (double)g.idzf[k] : 0.0;
  for (int e = tid; e < JT * nx; e += nthr) {
    int r = e / nx, i = e - r * nx, j = j0 + r;
    double val;
    if (u != nullptr) {
      const size_t o = pidx(k, j, i, ny, nx);
      val = ((double)u[o] - (double)u[pidx(k, j, wrap(i - 1, nx), ny, nx)]) * idx +
            ((double)v[o] - (double)v[pidx(k, wrap(j - 1, ny), i, ny, nx)]) * idy +
            ((double)w[pidx(k + 1, j, i, ny, nx)] - (double)w[o]) * idzf;
    } else {
      val = field[pidx(k, j, i, ny, nx)];
    }
    val *= scale;
    double* dst = reinterpret_cast<double*>(&b0[(r >> 1) * rs + padi<double>(i)]);
    dst[r & 1] = val;
  }
  __syncthreads();
  int which = fft_rows<double, false>(b0, b1, JT / 2, rs, plx, stw, tid, nthr);
  const cpx<double>* Z = which ? b1 : b0;
  for (int e = tid; e < nxh * JT; e += nthr) {
    int m = e / JT, r = e - m * JT, pr = r >> 1;
    cpx<double> Zm = Z[pr * rs + padi<double>(m)];
    cpx<double> Zn = cconj(Z[pr * rs + padi<double>(m == 0 ? 0 : nx - m)]);
    cpx<double> out;
    if ((r & 1) == 0) out = cscale(cadd(Zm, Zn), 0.5);
    else {
      cpx<double> d = csub(Zm, Zn);  // (Z - conj Z(-m)) / (2i) = -i/2 * d
      out = cmake<double>(0.5 * d.y, -0.5 * d.x);
    }
    X[((size_t)m * nz + k) * ny + j0 + r] = out;
  }
}

// In-place complex FFT along y of the rows X[kx][k][:] (RB rows per block).
template <bool INV>
__global__ void __launch_bounds__(256) k_ffty(cpx<double>* __restrict__ X, int nrows, int ny, FftPlan ply,
                                              const cpx<double>* __restrict__ twy, int RB) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int rs = padded_len<double>(ny);
  cpx<double>* b0 = reinterpret_cast<cpx<double>*>(smraw);
  cpx<double>* b1 = b0 + RB * rs;
  cpx<double>* stw = b1 + RB * rs;  // twiddles (ny)
  const int r0 = blockIdx.x * RB;
  const int nb = min(RB, nrows - r0);
  const int tid = threadIdx.x, nthr = blockDim.x;
  cpx<double>* base = X + (size_t)r0 * ny;
  stage_twiddles(stw, twy, ny, tid, nthr);
  for (int e = tid; e < nb * ny; e += nthr) {
    const int r = e / ny, jj = e - r * ny;
    b0[r * rs + padi<double>(jj)] = base[e];
  }
  __syncthreads();
  int which = fft_rows<double, INV>(b0, b1, nb, rs, ply, stw, tid, nthr);
  const cpx<double>* Z = which ? b1 : b0;
  for (int e = tid; e < nb * ny; e += nthr) {
    const int r = e / ny, jj = e - r * ny;
    base[e] = Z[r * rs + padi<double>(jj)];
  }
}

// In-place complex FFT along y of the rows X[kx][k][:] with the register
// transform (ny = N1 * 16): RowFft<N1>::RPW rows per warp, each row read and
// written once, no block barrier; warps stride over the rows, loading the
// next rows while transforming the current ones.
// Rows row0 .. row0+RPW-1 (< nrows) by one warp, as one pass of the
// k_ffty_reg loop below; `tiles` holds the warp's RPW transpose tiles.
template <int N1, bool INV>
__device__ __forceinline__ void ffty_rows(cpx<double>* __restrict__ X, int nrows, const cpx<double>* __restrict__ twy,
                                          int row0, cpx<double>* tiles) {
  using RF = RowFft<N1>;
  const int lane = threadIdx.x & 31;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;   // row of the warp, lane in the row
  cpx<double>* tile = tiles + (size_t)sub * RF::TILE;
  const int row = row0 + sub;
  const bool ok = sub < RF::RPW && row < nrows && TC_IN((size_t)row * RF::N, (size_t)nrows * RF::N, RF::N);
  cpx<double>* x = X + (size_t)(ok ? row : 0) * RF::N;
  if (ok && l < RF::N2) rowfft_pass1<N1, INV>([&](int e) { return x[e]; }, l, tile, twy);
  __syncwarp();
  if (ok && l < RF::N1) rowfft_pass2<N1, INV>([&](int e, cpx<double> val) { x[e] = val; }, l, tile);
  __syncwarp();
}

template <int N1, bool INV>
__global__ void __launch_bounds__(128) k_ffty_reg(cpx<double>* __restrict__ X, int nrows,
                                                 const cpx<double>* __restrict__ twy) {
  using RF = RowFft<N1>;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;   // row of the warp, lane in the row
  const int wpb = blockDim.x >> 5;
  cpx<double>* tile = reinterpret_cast<cpx<double>*>(smraw) + (size_t)(warp * RF::RPW + sub) * RF::TILE;
  const int rstep = gridDim.x * wpb * RF::RPW;
  // the next rows' values are loaded before this row's transform
  const bool lane_ld = sub < RF::RPW && l < RF::N2;
  int row0 = (blockIdx.x * wpb + warp) * RF::RPW;
  cpx<double> v[RF::N1];
  auto ldrow = [&](int r0, cpx<double> (&o)[RF::N1]) {
    const int row = r0 + sub;
    if (lane_ld && row < nrows && TC_IN((size_t)row * RF::N, (size_t)nrows * RF::N, RF::N)) {
      const cpx<double>* x = X + (size_t)row * RF::N;
#pragma unroll
      for (int n1 = 0; n1 < RF::N1; ++n1) o[n1] = x[RF::N2 * n1 + l];
    }
  };
  ldrow(row0, v);
  for (; row0 < nrows; row0 += rstep) {
    const int row = row0 + sub;
    const bool ok = sub < RF::RPW && row < nrows && TC_IN((size_t)row * RF::N, (size_t)nrows * RF::N, RF::N);
    cpx<double>* x = X + (size_t)(ok ? row : 0) * RF::N;
    cpx<double> vn[RF::N1];
    ldrow(row0 + rstep, vn);
    if (ok && l < RF::N2) rowfft_pass1_regs<N1, INV>(v, l, tile, twy);
    __syncwarp();
    if (ok && l < RF::N1) rowfft_pass2<N1, INV>([&](int e, cpx<double> val) { x[e] = val; }, l, tile);
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < RF::N1; ++n1) v[n1] = vn[n1];
  }
}

// Divergence (as k_div_fftx) of rows j0 .. j0+XR-1 of plane k and forward
// real FFT along x with the register transform (nx = N1 * 16); two real rows
// travel as one complex row, RowFft<N1>::RPW such rows per warp (XR / 2 / RPW
// warps a block).  The unpacked half spectra are written transposed,
// X[m][k][j], as in k_div_fftx.
// rows per block of the register x transforms (XR below)
#define XROWS 16

// Rows j0 = bx * XR .. of plane k; blockDim.x may exceed the warps the rows
// need (ensemble kernel), the extra warps only take part in the barrier.
// XT: element type of the written spectrum (double, or float for the
// single-precision Poisson step, which also subtracts lsub * lsub_scale: the
// base pressure's Laplacian).
template <class T, int N1, int XR, class XT = double>
__device__ __forceinline__ void fftx_tile(const Grid<T>& g, const T* __restrict__ u, const T* __restrict__ v,
                                          const T* __restrict__ w, const double* __restrict__ field,
                                          cpx<XT>* __restrict__ X, const cpx<double>* __restrict__ twx,
                                          double scale, int bx, int k, const float* __restrict__ lsub = nullptr,
                                          double lsub_scale = 0.0) {
  using RF = RowFft<N1>;
  constexpr int N = RF::N, NH = N / 2 + 1;
  constexpr int ZP = (RF::TILE + 7) / 8 * 8 + 1;          // row pitch of the spectra (16 B mod 128 B)
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<double>* zs = reinterpret_cast<cpx<double>*>(smraw);  // XR/2 packed rows x ZP
  const int ny = g.ny, nz = g.nz;
  const int j0 = bx * XR;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;
  const int pr = warp * RF::RPW + sub;                      // packed row: j = j0 + 2 pr, +1
  const bool ok = sub < RF::RPW && pr < XR / 2;
  cpx<double>* tile = zs + (size_t)(ok ? pr : 0) * ZP;
  const double idx = (double)g.idx, idy = (double)g.idy;
  const double idzf = (u != nullptr) ? (double)g.idzf[k] : 0.0;
  const int ja = j0 + 2 * pr, jb = ja + 1;
#ifdef TC_BOUNDS_CHECK
  const size_t ncell = (size_t)N * ny * nz, nface = (size_t)N * ny * (nz + 1);  // field extents
  auto divv = [&](int j, int i) -> double {
    double val;
    const size_t o = pidx(k, j, i, ny, N);
    if (u != nullptr) {
      const size_t oxm = pidx(k, j, i == 0 ? N - 1 : i - 1, ny, N), oym = pidx(k, j == 0 ? ny - 1 : j - 1, i, ny, N);
      const size_t ozp = pidx(k + 1, j, i, ny, N);
      if (!(TC_IN(o, ncell, 1) && TC_IN(oxm, ncell, 1) && TC_IN(oym, ncell, 1) && TC_IN(ozp, nface, 1))) return 0.0;
      val = ((double)u[o] - (double)u[oxm]) * idx + ((double)v[o] - (double)v[oym]) * idy +
            ((double)w[ozp] - (double)w[o]) * idzf;
    } else {
      if (!TC_IN(o, ncell, 1)) return 0.0;
      val = field[o];
    }
    if constexpr (sizeof(XT) == 4) return val * scale - (double)lsub[o] * lsub_scale;
    return val * scale;
  };
#else
  // (the checked form above measured 50% slower here even with its checks
  // compiled out, so the normal build keeps this form)
  auto divv = [&](int j, int i) -> double {
    double val;
    if (u != nullptr) {
      const size_t o = pidx(k, j, i, ny, N);
      val = ((double)u[o] - (double)u[pidx(k, j, i == 0 ? N - 1 : i - 1, ny, N)]) * idx +
            ((double)v[o] - (double)v[pidx(k, j == 0 ? ny - 1 : j - 1, i, ny, N)]) * idy +
            ((double)w[pidx(k + 1, j, i, ny, N)] - (double)w[o]) * idzf;
    } else {
      val = field[pidx(k, j, i, ny, N)];
    }
    if constexpr (sizeof(XT) == 4) return val * scale - (double)lsub[pidx(k, j, i, ny, N)] * lsub_scale;
    return val * scale;
  };
#endif
  if (ok && l < RF::N2)
    rowfft_pass1<N1, false>([&](int i) { return cmake<double>(divv(ja, i), divv(jb, i)); }, l, tile, twx);
  __syncwarp();
  cpx<double> b[RF::N2];
  if (ok && l < RF::N1) {
#pragma unroll
    for (int n2 = 0; n2 < RF::N2; ++n2) b[n2] = tile[l * RF::TP + n2];
  }
  __syncwarp();
  if (ok && l < RF::N1) {
    Dft<RF::N2, false>::run(b);
#pragma unroll
    for (int k2 = 0; k2 < RF::N2; ++k2) tile[l + RF::N1 * k2] = b[k2];  // Z[m], natural order
  }
  __syncthreads();
  // unpack: A = (Z[m] + conj Z[N-m]) / 2 (row ja), B = (Z[m] - conj Z[N-m]) / (2i) (row jb)
  for (int e = threadIdx.x; e < NH * XR; e += blockDim.x) {
    const int m = e / XR, r = e % XR, q = r >> 1;
    const cpx<double> Zm = zs[q * ZP + m];
    const cpx<double> Zn = cconj(zs[q * ZP + (m == 0 ? 0 : N - m)]);
    cpx<double> out;
    if ((r & 1) == 0) out = cscale(cadd(Zm, Zn), 0.5);
    else {
      const cpx<double> d = csub(Zm, Zn);
      out = cmake<double>(0.5 * d.y, -0.5 * d.x);
    }
    const size_t xo = ((size_t)m * nz + k) * ny + j0 + r;
    if (TC_IN(xo, (size_t)NH * nz * ny, 1)) X[xo] = cmake<XT>((XT)out.x, (XT)out.y);
  }
}

template <class T, int N1, int XR>
__global__ void __launch_bounds__(16 * XR / RowFft<N1>::RPW) k_div_fftx_reg(Grid<T> g, const T* __restrict__ u, const T* __restrict__ v,
                                                     const T* __restrict__ w, const double* __restrict__ field,
                                                     cpx<double>* __restrict__ X,
                                                     const cpx<double>* __restrict__ twx, double scale) {
  fftx_tile<T, N1, XR>(g, u, v, w, field, X, twx, scale, blockIdx.x, blockIdx.y);
}

// The x transform of the single-precision Poisson step: div(u**)/dt minus
// the base pressure's Laplacian lp (k_base_lap), in FP64 arithmetic, the
// spectrum written in FP32.
template <class T, int N1, int XR>
__global__ void __launch_bounds__(16 * XR / RowFft<N1>::RPW) k_div_fftx_reg32(Grid<T> g, const T* __restrict__ u,
                                                                             const T* __restrict__ v,
                                                                             const T* __restrict__ w,
                                                                             cpx<float>* __restrict__ X,
                                                                             const cpx<double>* __restrict__ twx,
                                                                             double scale,
                                                                             const float* __restrict__ lp,
                                                                             double lp_scale) {
  fftx_tile<T, N1, XR, float>(g, u, v, w, nullptr, X, twx, scale, blockIdx.x, blockIdx.y, lp, lp_scale);
}

// Inverse real FFT along x of rows j0 .. j0+XR-1 of plane k with the
// register transform (nx = N1 * 16); writes p[k][j][i] (FP64).  Two rows
// travel as one complex row Z = A + i B built from the half spectra (DC and
// Nyquist real).
// Row pitch of the staged half spectra of the inverse x transform: odd in
// 16-byte words, and two rows hold one transpose tile.
template <int N1> __host__ __device__ constexpr int ifftx_pitch() {
  constexpr int NH = RowFft<N1>::N / 2 + 1, HT = (RowFft<N1>::TILE + 1) / 2;
  return ((NH > HT ? NH : HT) + 7) / 8 * 8 + 1;
}

// XT / PT: element types of the spectrum read and of the field written
// (double / double, or float / float for the increment of the
// single-precision Poisson step; the transform itself runs in FP64).
template <int N1, int XR, class XT = double, class PT = double>
__device__ __forceinline__ void ifftx_tile(const cpx<XT>* __restrict__ X, PT* __restrict__ p, int ny, int nz,
                                           const cpx<double>* __restrict__ twx, int bx, int k) {
  using RF = RowFft<N1>;
  constexpr int N = RF::N, NH = N / 2 + 1;
  constexpr int SP = ifftx_pitch<N1>();                      // staging pitch
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<double>* S = reinterpret_cast<cpx<double>*>(smraw);   // XR rows x SP half spectra
  const int j0 = bx * XR;
  for (int e = threadIdx.x; e < NH * XR; e += blockDim.x) {
    const int m = e / XR, r = e % XR;
    const size_t xo = ((size_t)m * nz + k) * ny + j0 + r;
    const cpx<XT> x = TC_IN(xo, (size_t)NH * nz * ny, 1) ? X[xo] : cpx<XT>{};
    cpx<double> val = cmake<double>((double)x.x, (double)x.y);
    if (m == 0 || 2 * m == N) val.y = 0.0;  // irfft ignores these imaginary parts
    S[r * SP + m] = val;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;
  const int pr = warp * RF::RPW + sub;
  const bool ok = sub < RF::RPW && pr < XR / 2;
  // a packed row's transpose tile overlays the two staged rows it reads
  // (the warp reads them all before any lane writes its tile)
  const cpx<double>* A = S + (2 * (ok ? pr : 0)) * SP;
  const cpx<double>* B = A + SP;
  cpx<double>* tile = S + (2 * (ok ? pr : 0)) * SP;
  auto ld = [&](int m) -> cpx<double> {
    cpx<double> a, bb;
    if (m < NH) { a = A[m]; bb = B[m]; }
    else { a = cconj(A[N - m]); bb = cconj(B[N - m]); }
    return cmake<double>(a.x - bb.y, a.y + bb.x);  // A + i B
  };
  cpx<double> vr[RF::N1];
  if (ok && l < RF::N2) {
#pragma unroll
    for (int n1 = 0; n1 < RF::N1; ++n1) vr[n1] = ld(RF::N2 * n1 + l);
  }
  __syncwarp();
  if (ok && l < RF::N2) rowfft_pass1_regs<N1, true>(vr, l, tile, twx);
  __syncwarp();
  const size_t po = ((size_t)k * ny + j0 + 2 * (ok ? pr : 0)) * N;
  PT* pa = p + po;
  const size_t pn = (size_t)N * ny * nz;  // extent of p (bounds-checked builds)
  (void)pn;
  if (ok && l < RF::N1)
    rowfft_pass2<N1, true>([&](int i, cpx<double> z) {
      if (TC_IN(po + i, pn, 1) && TC_IN(po + N + i, pn, 1)) { pa[i] = (PT)z.x; pa[N + i] = (PT)z.y; }
    }, l, tile);
}

template <int N1, int XR>
__global__ void __launch_bounds__(16 * XR / RowFft<N1>::RPW) k_ifftx_reg(const cpx<double>* __restrict__ X, double* __restrict__ p,
                                                  int ny, int nz, const cpx<double>* __restrict__ twx) {
  ifftx_tile<N1, XR>(X, p, ny, nz, twx, blockIdx.x, blockIdx.y);
}

// Inverse x transform of the single-precision Poisson step: FP32 spectrum
// in, FP64 transform, FP32 pressure increment out.
template <int N1, int XR>
__global__ void __launch_bounds__(16 * XR / RowFft<N1>::RPW) k_ifftx_reg32(const cpx<float>* __restrict__ X,
                                                                          float* __restrict__ dp, int ny, int nz,
                                                                          const cpx<double>* __restrict__ twx) {
  ifftx_tile<N1, XR, float, float>(X, dp, ny, nz, twx, blockIdx.x, blockIdx.y);
}

// Thomas sweep along z for every mode (kx, ky), one thread per mode
// (projection_fft.py:167-215), with the tridiagonal rows of
// projection_fft.py:44-82 built on the fly.  The (0,0) mode is singular: its
// last unknown is pinned to 0 (explicit gauge) instead of dividing by the
// roundoff-level pivot.  FP64; d' in place in X, c' in shared memory.  Loads
// are issued TRI_B levels ahead of the dependent recurrence.
#define TRI_B 32
__global__ void __launch_bounds__(64) k_tri(cpx<double>* __restrict__ X, PoissonTabs tb, int nxh, int ny, int nz) {
  extern __shared__ double cps[];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxh * ny) return;
  const int kx = t / ny, ky = t - kx * ny;
  const double K2 = tb.k2x[kx] + tb.k2y[ky];
  const size_t stride = ny;
  cpx<double>* col = X + (size_t)kx * nz * ny + ky;
  const int bt = blockDim.x;
  double* cpl = cps + threadIdx.x;
  cpx<double> buf[TRI_B];
  // forward
  double dpr = 0.0, dpi = 0.0, cprev = 0.0;
  for (int k0 = 0; k0 < nz; k0 += TRI_B) {
#pragma unroll
    for (int b = 0; b < TRI_B; ++b)
      if (k0 + b < nz) buf[b] = col[(size_t)(k0 + b) * stride];
#pragma unroll
    for (int b = 0; b < TRI_B; ++b) {
      const int k = k0 + b;
      if (k < nz) {
        const double cl = tb.cl[k], cr = tb.cr[k];
        const double a = (k == 0) ? 0.0 : cl;
        double bb = -(cl + cr + K2);
        if (k == 0) bb += cl;
        if (k == nz - 1) bb += cr;
        const double c = (k == nz - 1) ? 0.0 : cr;
        const double rden = 1.0 / (bb - a * cprev);
        const double cpk = c * rden;
        dpr = (buf[b].x - a * dpr) * rden;
        dpi = (buf[b].y - a * dpi) * rden;
        cpl[(size_t)k * bt] = cpk;
        cprev = cpk;
        col[(size_t)k * stride] = cpx<double>{dpr, dpi};
      }
    }
  }
  // backward
  double xr = dpr, xi = dpi;
  if (kx == 0 && ky == 0) { xr = 0.0; xi = 0.0; }
  col[(size_t)(nz - 1) * stride] = cpx<double>{xr, xi};
  for (int k1 = nz - 2; k1 >= 0; k1 -= TRI_B) {
#pragma unroll
    for (int b = 0; b < TRI_B; ++b)
      if (k1 - b >= 0) buf[b] = col[(size_t)(k1 - b) * stride];
#pragma unroll
    for (int b = 0; b < TRI_B; ++b) {
      const int k = k1 - b;
      if (k >= 0) {
        const double cpk = cpl[(size_t)k * bt];
        xr = buf[b].x - cpk * xr;
        xi = buf[b].y - cpk * xi;
        col[(size_t)k * stride] = cpx<double>{xr, xi};
      }
    }
  }
}

// LU factors of every mode's z system, computed once per grid: the rows of
// projection_fft.py:44-82 do not depend on dt or on the data, so
// rden[k] = 1/(b_k - a_k c'_{k-1}) and c'_k = c_k rden[k] are tabulated in the
// layout of X ([kx][k][ky]) with the same arithmetic as the sweep of k_tri.
__global__ void __launch_bounds__(128) k_tri_factors(PoissonTabs tb, double* __restrict__ rden_t,
                                                     double* __restrict__ cp_t, int nxh, int ny, int nz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxh * ny) return;
  const int kx = t / ny, ky = t - kx * ny;
  const double K2 = tb.k2x[kx] + tb.k2y[ky];
  const size_t base = (size_t)kx * nz * ny + ky;
  double cprev = 0.0;
  for (int k = 0; k < nz; ++k) {
    const double cl = tb.cl[k], cr = tb.cr[k];
    const double a = (k == 0) ? 0.0 : cl;
    double bb = -(cl + cr + K2);
    if (k == 0) bb += cl;
    if (k == nz - 1) bb += cr;
    const double c = (k == nz - 1) ? 0.0 : cr;
    const double rden = 1.0 / (bb - a * cprev);
    const double cpk = c * rden;
    rden_t[base + (size_t)k * ny] = rden;
    cp_t[base + (size_t)k * ny] = cpk;
    cprev = cpk;
  }
}

// Division-free Thomas sweep with the tabulated factors: forward
// d'_k = (d_k - a_k d'_{k-1}) rden_k, backward x_k = d'_k - c'_k x_{k+1}, the
// (0,0) mode gauged (x_{nz-1} = 0).  One thread per mode; the next TRIF_B
// levels are in flight while the current ones are used.
#define TRIF_B 16
__global__ void __launch_bounds__(128) k_tri_lu(cpx<double>* __restrict__ X, const double* __restrict__ rden_t,
                                                const double* __restrict__ cp_t, PoissonTabs tb, int nxh, int ny,
                                                int nz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxh * ny) return;
  const int kx = t / ny, ky = t - kx * ny;
  const size_t base = (size_t)kx * nz * ny + ky;
  cpx<double>* col = X + base;
  const double* rd = rden_t + base;
  const double* cpt = cp_t + base;
  const size_t st = ny;
  cpx<double> dc[TRIF_B], dn[TRIF_B];
  double fc[TRIF_B], fn[TRIF_B];
#pragma unroll
  for (int b = 0; b < TRIF_B; ++b) {
    if (b < nz) { dc[b] = col[(size_t)b * st]; fc[b] = ldg(rd + (size_t)b * st); }
  }
  double dpr = 0.0, dpi = 0.0;
  for (int k0 = 0; k0 < nz; k0 += TRIF_B) {
#pragma unroll
    for (int b = 0; b < TRIF_B; ++b) {
      const int kk = k0 + TRIF_B + b;
      if (kk < nz) { dn[b] = col[(size_t)kk * st]; fn[b] = ldg(rd + (size_t)kk * st); }
    }
#pragma unroll
    for (int b = 0; b < TRIF_B; ++b) {
      const int k = k0 + b;
      if (k < nz) {
        const double a = (k == 0) ? 0.0 : tb.cl[k];
        dpr = (dc[b].x - a * dpr) * fc[b];
        dpi = (dc[b].y - a * dpi) * fc[b];
        col[(size_t)k * st] = cpx<double>{dpr, dpi};
      }
    }
#pragma unroll
    for (int b = 0; b < TRIF_B; ++b) { dc[b] = dn[b]; fc[b] = fn[b]; }
  }
  double xr = dpr, xi = dpi;
  if (kx == 0 && ky == 0) { xr = 0.0; xi = 0.0; }
  col[(size_t)(nz - 1) * st] = cpx<double>{xr, xi};
#pragma unroll
  for (int b = 0; b < TRIF_B; ++b) {
    const int k = nz - 2 - b;
    if (k >= 0) { dc[b] = col[(size_t)k * st]; fc[b] = ldg(cpt + (size_t)k * st); }
  }
  for (int k1 = nz - 2; k1 >= 0; k1 -= TRIF_B) {
#pragma unroll
    for (int b = 0; b < TRIF_B; ++b) {
      const int k = k1 - TRIF_B - b;
      if (k >= 0) { dn[b] = col[(size_t)k * st]; fn[b] = ldg(cpt + (size_t)k * st); }
    }
#pragma unroll
    for (int b = 0; b < TRIF_B; ++b) {
      const int k = k1 - b;
      if (k >= 0) {
        xr = dc[b].x - fc[b] * xr;
        xi = dc[b].y - fc[b] * xi;
        col[(size_t)k * st] = cpx<double>{xr, xi};
      }
    }
#pragma unroll
    for (int b = 0; b < TRIF_B; ++b) { dc[b] = dn[b]; fc[b] = fn[b]; }
  }
}

// Batched in-place FFT of `nr` padded rows of R, FB rows at a time through
// the scratch rows S (the Stockham passes alternate between the two).
template <bool INV>
__device__ __forceinline__ void yz_fft_rows(cpx<double>* R, cpx<double>* S, int nr, int FB, int rs, int ny,
                                            const FftPlan& ply, const cpx<double>* tw, int tid, int nthr) {
  for (int b0 = 0; b0 < nr; b0 += FB) {
    const int nb = min(FB, nr - b0);
    cpx<double>* A = R + (size_t)b0 * rs;
    if (fft_rows<double, INV>(A, S, nb, rs, ply, tw, tid, nthr)) {
      for (int e = tid; e < nb * ny; e += nthr) {
        const int r = e / ny, j = e - r * ny;
        A[r * rs + padi<double>(j)] = S[r * rs + padi<double>(j)];
      }
      __syncthreads();
    }
  }
}

// c' of every mode's z system at the last level below each chunk of P
// levels (k = r P - 1, r = 1 .. CS-1), with the arithmetic of k_tri_factors
// so that k_yz_solve's on-the-fly factors equal the tabulated ones bit for
// bit.  Layout cpb[kx][r][ky]; r = 0 holds 0 (no level below the first
// chunk).
__global__ void __launch_bounds__(128) k_tri_chunk_cp(PoissonTabs tb, double* __restrict__ cpb, int nxh, int ny,
                                                      int nz, int CS, int P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxh * ny) return;
  const int kx = t / ny, ky = t - kx * ny;
  const double K2 = tb.k2x[kx] + tb.k2y[ky];
  double* out = cpb + (size_t)kx * CS * ny + ky;
  out[0] = 0.0;
  double cprev = 0.0;
  for (int k = 0; k < nz; ++k) {
    const double cl = tb.cl[k], cr = tb.cr[k];
    const double a = (k == 0) ? 0.0 : cl;
    double bb = -(cl + cr + K2);
    if (k == 0) bb += cl;
    if (k == nz - 1) bb += cr;
    const double c = (k == nz - 1) ? 0.0 : cr;
    const double rden = 1.0 / (bb - a * cprev);
    cprev = c * rden;
    if ((k + 1) % P == 0 && (k + 1) / P < CS) out[(size_t)((k + 1) / P) * ny] = cprev;
  }
  for (int r = (nz + P - 1) / P; r < CS; ++r) out[(size_t)r * ny] = 0.0;  // empty chunks
}

// Fused middle of the Poisson solve: [FFT along y] -> [Thomas along z] ->
// [inverse FFT along y] of one kx slab X[kx][:][:] per thread-block cluster
// of CS CTAs, so the spectrum crosses HBM once each way instead of three
// times and no factor table is read.  CTA r of the cluster holds planes
// [r P, r P + P) of the slab in shared memory (padded rows); one thread per
// column ky sweeps both parts of its chunk.  The LU factors
// (rden_k = 1/(b_k - a_k c'_{k-1}), c'_k = c_k rden_k, projection_fft.py:44-82
// rows) are rebuilt on the fly from c' below the chunk (k_tri_chunk_cp) and
// kept in registers.  The chunk is swept forward from a zero boundary value;
// the chunk ends, with the chunk products G = prod (-a_k rden_k), are read
// from the lower CTAs through distributed shared memory and scanned into
// d'(start-1), and the backward sweep adds G_k d'(start-1) (G_k the product
// from the chunk start to k) to each forward value; the backward pass is
// stitched the same way with H = prod (-c'_k) and x(end+1) from the upper
// CTAs.  The (0,0) mode is gauged as in k_tri_lu (x_{nz-1} = 0); its singular
// last pivot is never used.  Every CTA takes the same three cluster barriers;
// the last keeps each CTA's shared memory alive until no peer reads it.
template <int PM>
__global__ void __launch_bounds__(512) k_yz_solve(cpx<double>* __restrict__ X, const double* __restrict__ cpb,
                                                  PoissonTabs tb, FftPlan ply, const cpx<double>* __restrict__ twy,
                                                  int ny, int nz, int P, int FB) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smraw[];
  const int CS = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int kx = blockIdx.x / CS;
  const int rs = padded_len<double>(ny);
  cpx<double>* R = reinterpret_cast<cpx<double>*>(smraw);    // P rows
  cpx<double>* S = R + (size_t)P * rs;                         // FB scratch rows
  cpx<double>* tw = S + (size_t)FB * rs;                       // ny twiddles
  cpx<double>* eV = tw + ny;                                   // ny: forward chunk-end values
  cpx<double>* sZ = eV + ny;                                   // ny: backward chunk-start values
  double* eG = reinterpret_cast<double*>(sZ + ny);             // ny: forward chunk products
  double* sH = eG + ny;                                        // ny: backward chunk products
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int k0 = rank * P;
  const int nr = max(0, min(P, nz - k0));
  cpx<double>* slab = X + ((size_t)kx * nz + k0) * ny;
  stage_twiddles(tw, twy, ny, tid, nthr);
#pragma unroll 4
  for (int e = tid; e < nr * ny; e += nthr) {
    const int r = e / ny, j = e - r * ny;
    R[r * rs + padi<double>(j)] = slab[e];
  }
  __syncthreads();
  yz_fft_rows<false>(R, S, nr, FB, rs, ny, ply, tw, tid, nthr);

  // one column per thread (blockDim >= ny); factors in registers
  const int j = tid;
  const bool colt = j < ny;
  const double K2 = colt ? tb.k2x[kx] + tb.k2y[j] : 0.0;
  double cpv[PM], gv[PM];
  cpx<double>* col = R + (colt ? padi<double>(j) : 0);
  if (colt) {
    double cprev = cpb[((size_t)kx * CS + rank) * ny + j];
    double yr = 0.0, yi = 0.0, g = 1.0;
#pragma unroll
    for (int r = 0; r < PM; ++r) {
      if (r < nr) {
        const int k = k0 + r;
        const double cl = tb.cl[k], cr = tb.cr[k];
        const double a = (k == 0) ? 0.0 : cl;
        double bb = -(cl + cr + K2);
        if (k == 0) bb += cl;
        if (k == nz - 1) bb += cr;
        const double c = (k == nz - 1) ? 0.0 : cr;
        const double rd = 1.0 / (bb - a * cprev);
        const double cpk = (k == nz - 1) ? 0.0 : c * rd;  // last level: c = 0 (never 0 * inf)
        const cpx<double> d = col[r * rs];
        yr = (d.x - a * yr) * rd;
        yi = (d.y - a * yi) * rd;
        col[r * rs] = cpx<double>{yr, yi};
        g *= -a * rd;
        gv[r] = g;
        cpv[r] = cpk;
        cprev = cpk;
      }
    }
    eV[j] = cpx<double>{yr, yi};
    eG[j] = g;
  }
  cluster.sync();
  if (colt) {
    // true d'(start-1) from the lower chunks
    double dr = 0.0, di = 0.0;
    for (int c = 0; c < rank; ++c) {
      const cpx<double> v = *cluster.map_shared_rank(eV + j, c);
      const double gg = *cluster.map_shared_rank(eG + j, c);
      dr = v.x + gg * dr;
      di = v.y + gg * di;
    }
    const bool gauge = (kx == 0) && (j == 0);
    double zr = 0.0, zi = 0.0, h = 1.0;
#pragma unroll
    for (int r = PM - 1; r >= 0; --r) {
      if (r < nr) {
        const int k = k0 + r;
        const cpx<double> y = col[r * rs];
        double vr = y.x + gv[r] * dr, vi = y.y + gv[r] * di;
        if (gauge && k == nz - 1) { vr = 0.0; vi = 0.0; }
        zr = vr - cpv[r] * zr;
        zi = vi - cpv[r] * zi;
        col[r * rs] = cpx<double>{zr, zi};
        h *= -cpv[r];
        gv[r] = h;  // H_k from here on
      }
    }
    sZ[j] = cpx<double>{zr, zi};
    sH[j] = h;
  }
  cluster.sync();
  if (colt) {
    // true x(end+1) from the upper chunks; x_k = z_k + H_k x(end+1)
    double xr = 0.0, xi = 0.0;
    for (int c = CS - 1; c > rank; --c) {
      const cpx<double> v = *cluster.map_shared_rank(sZ + j, c);
      const double hh = *cluster.map_shared_rank(sH + j, c);
      xr = v.x + hh * xr;
      xi = v.y + hh * xi;
    }
#pragma unroll
    for (int r = 0; r < PM; ++r) {
      if (r < nr) {
        const cpx<double> z = col[r * rs];
        col[r * rs] = cpx<double>{z.x + gv[r] * xr, z.y + gv[r] * xi};
      }
    }
  }
  cluster.barrier_arrive();  // this CTA reads no peer memory after here
  __syncthreads();
  yz_fft_rows<true>(R, S, nr, FB, rs, ny, ply, tw, tid, nthr);
#pragma unroll 4
  for (int e = tid; e < nr * ny; e += nthr) {
    const int r = e / ny, jj = e - r * ny;
    slab[e] = R[r * rs + padi<double>(jj)];
  }
  cluster.barrier_wait();
}

// k_tri_lu with the real and imaginary parts of a mode on two threads (the
// factors are real, so the two recurrences are independent): twice the
// threads in flight, half the registers per level, TRIP_B levels prefetched.
#define TRIP_B 16

// The sweeps of tri_lu2_thread for nz a multiple of 2 LB (LB levels per
// block), with the same arithmetic: 32-bit running offsets (one multiply-add
// per address), the level coefficients at constant offsets from a block's
// first level, no per-level guards, and two prefetch buffers used in turn
// instead of one that is shifted.  Integer work was most of the general form's instructions, and
// with two warps per scheduler each level costs its instructions' latencies.
// The backward sweep starts at level nz-1 (x = d' there) so that it too
// covers whole blocks; the gauged (0,0) mode has 0 stored there first.
template <int LB>
__device__ __forceinline__ void tri_lu2_lean(double* __restrict__ col, const double* __restrict__ rd,
                                             const double* __restrict__ cpt, const double* __restrict__ cl,
                                             unsigned st, int nz, bool gauge, size_t lim, size_t tlim) {
  // lim / tlim: elements of X from col and of a table from rd / cpt (bounds-checked builds)
  (void)lim; (void)tlim;
  const unsigned st2 = 2u * st;
  double da[LB], fa[LB], db[LB], fb[LB];
  // levels k0 .. k0+LB-1 of d and of a factor table
  auto load_up = [&](double (&d)[LB], double (&f)[LB], const double* __restrict__ tab, int k0) {
    unsigned o = (unsigned)k0 * st2, q = (unsigned)k0 * st;
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      d[b] = TC_IN(o, lim, 1) ? col[o] : 0.0;
      f[b] = TC_IN(q, tlim, 1) ? ldg(tab + q) : 0.0;
      o += st2;
      q += st;
    }
  };
  // levels k1, k1-1, .. k1-LB+1
  auto load_dn = [&](double (&d)[LB], double (&f)[LB], const double* __restrict__ tab, int k1) {
    unsigned o = (unsigned)k1 * st2, q = (unsigned)k1 * st;
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      d[b] = TC_IN(o, lim, 1) ? col[o] : 0.0;
      f[b] = TC_IN(q, tlim, 1) ? ldg(tab + q) : 0.0;
      o -= st2;
      q -= st;
    }
  };
  double dp = 0.0;
  auto sweep_up = [&](const double (&d)[LB], const double (&f)[LB], int k0) {
    unsigned o = (unsigned)k0 * st2;
    const double* a = cl + k0;
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      const double ak = (b == 0 && k0 == 0) ? 0.0 : (TC_IN(k0 + b, nz, 1) ? ldg(a + b) : 0.0);
      dp = fma(-(ak * f[b]), dp, d[b] * f[b]);
      if (TC_IN(o, lim, 1)) col[o] = dp;
      o += st2;
    }
  };
  load_up(da, fa, rd, 0);
  for (int k0 = 0; k0 < nz; k0 += 2 * LB) {
    load_up(db, fb, rd, k0 + LB);
    sweep_up(da, fa, k0);
    if (k0 + 2 * LB < nz) load_up(da, fa, rd, k0 + 2 * LB);
    sweep_up(db, fb, k0 + LB);
  }
  if (gauge && TC_IN((unsigned)(nz - 1) * st2, lim, 1)) col[(unsigned)(nz - 1) * st2] = 0.0;
  double x = 0.0;
  auto sweep_dn = [&](const double (&d)[LB], const double (&f)[LB], int k1) {
    unsigned o = (unsigned)k1 * st2;
#pragma unroll
    for (int b = 0; b < LB; ++b) {
      // level nz-1 is d' itself: its table entry c_{nz-1} rden_{nz-1} is 0,
      // or not finite for the singular (0,0) mode
      x = (b == 0 && k1 == nz - 1) ? d[b] : d[b] - f[b] * x;
      if (TC_IN(o, lim, 1)) col[o] = x;
      o -= st2;
    }
  };
  load_dn(da, fa, cpt, nz - 1);
  for (int k1 = nz - 1; k1 >= 0; k1 -= 2 * LB) {
    load_dn(db, fb, cpt, k1 - LB);
    sweep_dn(da, fa, k1);
    if (k1 - 2 * LB >= 0) load_dn(da, fa, cpt, k1 - 2 * LB);
    sweep_dn(db, fb, k1 - LB);
  }
}

// Thread t of the sweep (mode t / 2, part t % 2); LEAN_B > 0: tri_lu2_lean
// with LEAN_B levels per block where nz is a multiple of 2 LEAN_B.
template <int LEAN_B>
__device__ __forceinline__ void tri_lu2_thread(double* __restrict__ Xd, const double* __restrict__ rden_t,
                                               const double* __restrict__ cp_t, const PoissonTabs& tb, int nxh,
                                               int ny, int nz, int t) {
  const int mode = t >> 1, part = t & 1;
  if (mode >= nxh * ny) return;
  const int kx = mode / ny, ky = mode - kx * ny;
  const size_t base = (size_t)kx * nz * ny + ky;
  double* col = Xd + 2 * base + part;
  const double* rd = rden_t + base;
  const double* cpt = cp_t + base;
  const size_t tlim = (size_t)nxh * nz * ny - base, lim = 2 * tlim - part;  // extents (bounds-checked builds)
  (void)tlim; (void)lim;
  if constexpr (LEAN_B > 0) {
    if (nz % (2 * LEAN_B) == 0) {
      tri_lu2_lean<LEAN_B>(col, rd, cpt, tb.cl, (unsigned)ny, nz, kx == 0 && ky == 0, lim, tlim);
      return;
    }
  }
  const size_t st = ny, st2 = 2 * (size_t)ny;
  double dc[TRIP_B], dn[TRIP_B], fc[TRIP_B], fn[TRIP_B];
#pragma unroll
  for (int b = 0; b < TRIP_B; ++b) {
    if (b < nz && TC_IN((size_t)b * st2, lim, 1) && TC_IN((size_t)b * st, tlim, 1)) {
      dc[b] = col[(size_t)b * st2];
      fc[b] = ldg(rd + (size_t)b * st);
    }
  }
  double dp = 0.0;
  for (int k0 = 0; k0 < nz; k0 += TRIP_B) {
#pragma unroll
    for (int b = 0; b < TRIP_B; ++b) {
      const int kk = k0 + TRIP_B + b;
      if (kk < nz && TC_IN((size_t)kk * st2, lim, 1) && TC_IN((size_t)kk * st, tlim, 1)) {
        dn[b] = col[(size_t)kk * st2];
        fn[b] = ldg(rd + (size_t)kk * st);
      }
    }
#pragma unroll
    for (int b = 0; b < TRIP_B; ++b) {
      const int k = k0 + b;
      if (k < nz) {
        // d'_k = (d_k - a_k d'_{k-1}) rden_k with the products formed off the
        // recurrence: one dependent FMA per level
        const double a = (k == 0) ? 0.0 : tb.cl[k];
        dp = fma(-(a * fc[b]), dp, dc[b] * fc[b]);
        if (TC_IN((size_t)k * st2, lim, 1)) col[(size_t)k * st2] = dp;
      }
    }
#pragma unroll
    for (int b = 0; b < TRIP_B; ++b) { dc[b] = dn[b]; fc[b] = fn[b]; }
  }
  double x = dp;
  if (kx == 0 && ky == 0) x = 0.0;
  if (TC_IN((size_t)(nz - 1) * st2, lim, 1)) col[(size_t)(nz - 1) * st2] = x;
#pragma unroll
  for (int b = 0; b < TRIP_B; ++b) {
    const int k = nz - 2 - b;
    if (k >= 0 && TC_IN((size_t)k * st2, lim, 1) && TC_IN((size_t)k * st, tlim, 1)) {
      dc[b] = col[(size_t)k * st2];
      fc[b] = ldg(cpt + (size_t)k * st);
    }
  }
  for (int k1 = nz - 2; k1 >= 0; k1 -= TRIP_B) {
#pragma unroll
    for (int b = 0; b < TRIP_B; ++b) {
      const int k = k1 - TRIP_B - b;
      if (k >= 0 && TC_IN((size_t)k * st2, lim, 1) && TC_IN((size_t)k * st, tlim, 1)) {
        dn[b] = col[(size_t)k * st2];
        fn[b] = ldg(cpt + (size_t)k * st);
      }
    }
#pragma unroll
    for (int b = 0; b < TRIP_B; ++b) {
      const int k = k1 - b;
      if (k >= 0) {
        x = dc[b] - fc[b] * x;
        if (TC_IN((size_t)k * st2, lim, 1)) col[(size_t)k * st2] = x;
      }
    }
#pragma unroll
    for (int b = 0; b < TRIP_B; ++b) { dc[b] = dn[b]; fc[b] = fn[b]; }
  }
}

// LEAN_B = 16 holds 254 registers (4 blocks per SM), LEAN_B = 8 166 (6):
// the deeper form where the whole launch is resident at once.
template <int LEAN_B>
__global__ void __launch_bounds__(64) k_tri_lu2(double* __restrict__ Xd, const double* __restrict__ rden_t,
                                                 const double* __restrict__ cp_t, PoissonTabs tb, int nxh, int ny,
                                                 int nz) {
  tri_lu2_thread<LEAN_B>(Xd, rden_t, cp_t, tb, nxh, ny, nz, blockIdx.x * blockDim.x + threadIdx.x);
}

// The Poisson middle in two streaming passes over the spectrum instead of
// three (register row transforms, tabulated LU factors):
//   k_ffty_fwd:  FFT along y of the rows X[kx][k][:] of one kx slab, then the
//                forward elimination d'_k = (d_k - a_k d'_{k-1}) rden_k of its
//                modes' z systems, d' written over X;
//   k_bwd_iffty: back substitution x_k = d'_k - c'_k x_{k+1} from the top
//                level down (x_{nz-1} = d'_{nz-1}; the gauged (0,0) mode has
//                d'_{nz-1} = 0 stored), then the inverse FFT along y.
// One CTA per kx slab walks it in groups of R = 8 RowFft::RPW rows: the 8
// warps transform R rows through shared-memory slots (a slot is a row's
// transpose tile, then the row in natural order), and thread t sweeps the
// columns ky = t, t + 256, .. of the group's levels (real and imaginary part
// together: the factors are real).  The next group's rows and factors are in
// flight while this group is transformed and swept.  Same arithmetic as
// k_ffty_reg + k_tri_lu2 + k_ffty_reg<inv>, so the results are bitwise the
// same; the spectrum crosses HBM twice less.
template <int N1> struct YzPass {
  using RF = RowFft<N1>;
  static constexpr int N = RF::N;
  static constexpr int NT = 256;                              // threads
  static constexpr int R = (NT / 32) * RF::RPW;               // rows per group
  static constexpr int SP = RF::TILE;                         // slot pitch (complex), >= N
  static constexpr int CPT = (N + NT - 1) / NT;               // sweep columns per thread
  static __host__ __device__ constexpr size_t smem() { return (size_t)R * SP * sizeof(cpx<double>); }
};

template <int N1>
__global__ void __launch_bounds__(256, 1) k_ffty_fwd(cpx<double>* __restrict__ X, const double* __restrict__ rden_t,
                                                     const double* __restrict__ cl,
                                                     const cpx<double>* __restrict__ twy, int nz) {
  using P = YzPass<N1>;
  using RF = typename P::RF;
  constexpr int N = P::N, R = P::R, SP = P::SP, CPT = P::CPT;
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<double>* slots = reinterpret_cast<cpx<double>*>(smraw);
  const int kx = blockIdx.x, tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;
  const int wr = warp * RF::RPW + sub;                        // the lane's row of a group
  const bool rl = sub < RF::RPW;
  cpx<double>* slab = X + (size_t)kx * nz * N;
  const double* rd = rden_t + (size_t)kx * nz * N;
  cpx<double>* tile = slots + (size_t)(rl ? wr : 0) * SP;
  cpx<double> v[RF::N1];
  auto ldrow = [&](int k0, cpx<double> (&o)[RF::N1]) {
    const int k = k0 + wr;
    if (rl && l < RF::N2 && k < nz && TC_IN((size_t)k * N, (size_t)nz * N, N)) {
      const cpx<double>* x = slab + (size_t)k * N;
#pragma unroll
      for (int n1 = 0; n1 < RF::N1; ++n1) o[n1] = x[RF::N2 * n1 + l];
    }
  };
  double dr[CPT], di[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) { dr[c] = 0.0; di[c] = 0.0; }
  const bool gauge_thread = kx == 0 && tid == 0;  // column ky = 0 of slab 0: the (0,0) mode
  ldrow(0, v);
  for (int k0 = 0; k0 < nz; k0 += R) {
    // this group's factors (used after the transform)
    double f[CPT][R];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int ky = tid + c * P::NT;
#pragma unroll
      for (int b = 0; b < R; ++b)
        f[c][b] = (ky < N && k0 + b < nz && TC_IN((size_t)(k0 + b) * N + ky, (size_t)nz * N, 1))
                      ? ldg(rd + (size_t)(k0 + b) * N + ky)
                      : 0.0;
    }
    cpx<double> vn[RF::N1];
    ldrow(k0 + R, vn);
    const bool rowok = rl && k0 + wr < nz;
    if (rowok && l < RF::N2) rowfft_pass1_regs<N1, false>(v, l, tile, twy);
    __syncwarp();
    cpx<double> bq[RF::N2];
    if (rowok && l < RF::N1) {
#pragma unroll
      for (int n2 = 0; n2 < RF::N2; ++n2) bq[n2] = tile[l * RF::TP + n2];
    }
    __syncwarp();
    if (rowok && l < RF::N1) {
      Dft<RF::N2, false>::run(bq);
#pragma unroll
      for (int k2 = 0; k2 < RF::N2; ++k2) tile[l + RF::N1 * k2] = bq[k2];  // the row in natural order
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int ky = tid + c * P::NT;
      if (ky < N) {
#pragma unroll
        for (int b = 0; b < R; ++b) {
          const int k = k0 + b;
          if (k < nz) {
            const double a = (k == 0) ? 0.0 : (TC_IN(k, nz, 1) ? ldg(cl + k) : 0.0);
            const cpx<double> d = slots[b * SP + ky];
            dr[c] = fma(-(a * f[c][b]), dr[c], d.x * f[c][b]);
            di[c] = fma(-(a * f[c][b]), di[c], d.y * f[c][b]);
            const bool g0 = gauge_thread && c == 0 && k == nz - 1;
            if (TC_IN((size_t)k * N + ky, (size_t)nz * N, 1))
              slab[(size_t)k * N + ky] = g0 ? cmake<double>(0.0, 0.0) : cmake<double>(dr[c], di[c]);
          }
        }
      }
    }
    __syncthreads();  // the slots are free for the next group
#pragma unroll
    for (int n1 = 0; n1 < RF::N1; ++n1) v[n1] = vn[n1];
  }
}

template <int N1>
__global__ void __launch_bounds__(256, 1) k_bwd_iffty(cpx<double>* __restrict__ X, const double* __restrict__ cp_t,
                                                      const cpx<double>* __restrict__ twy, int nz) {
  using P = YzPass<N1>;
  using RF = typename P::RF;
  constexpr int N = P::N, R = P::R, SP = P::SP, CPT = P::CPT;
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<double>* slots = reinterpret_cast<cpx<double>*>(smraw);
  const int kx = blockIdx.x, tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;
  const int wr = warp * RF::RPW + sub;
  const bool rl = sub < RF::RPW;
  cpx<double>* slab = X + (size_t)kx * nz * N;
  const double* cpt = cp_t + (size_t)kx * nz * N;
  cpx<double>* tile = slots + (size_t)(rl ? wr : 0) * SP;
  // a group is the levels k1, k1-1, .. k1-R+1 (slot b holds level k1 - b)
  cpx<double> d[CPT][R];
  double f[CPT][R];
  auto ldgrp = [&](int k1, cpx<double> (&dd)[CPT][R], double (&ff)[CPT][R]) {
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int ky = tid + c * P::NT;
#pragma unroll
      for (int b = 0; b < R; ++b) {
        const int k = k1 - b;
        const bool ok = ky < N && k >= 0 && TC_IN((size_t)k * N + ky, (size_t)nz * N, 1);
        dd[c][b] = ok ? slab[(size_t)k * N + ky] : cmake<double>(0.0, 0.0);
        ff[c][b] = ok ? ldg(cpt + (size_t)k * N + ky) : 0.0;
      }
    }
  };
  double xr[CPT], xi[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) { xr[c] = 0.0; xi[c] = 0.0; }
  ldgrp(nz - 1, d, f);
  for (int k1 = nz - 1; k1 >= 0; k1 -= R) {
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const int ky = tid + c * P::NT;
      if (ky < N) {
#pragma unroll
        for (int b = 0; b < R; ++b) {
          const int k = k1 - b;
          if (k >= 0) {
            // level nz-1 is d' itself: its factor c_{nz-1} rden_{nz-1} is 0,
            // or not finite for the singular (0,0) mode
            if (k == nz - 1) { xr[c] = d[c][b].x; xi[c] = d[c][b].y; }
            else { xr[c] = d[c][b].x - f[c][b] * xr[c]; xi[c] = d[c][b].y - f[c][b] * xi[c]; }
            slots[b * SP + ky] = cmake<double>(xr[c], xi[c]);
          }
        }
      }
    }
    __syncthreads();
    if (k1 - R >= 0) ldgrp(k1 - R, d, f);  // the next group's d' and factors, in flight during the transform
    const int k = k1 - wr;
    const bool rowok = rl && k >= 0 && TC_IN((size_t)k * N, (size_t)nz * N, N);
    cpx<double> vr[RF::N1];
    if (rowok && l < RF::N2) {
#pragma unroll
      for (int n1 = 0; n1 < RF::N1; ++n1) vr[n1] = tile[RF::N2 * n1 + l];
    }
    __syncwarp();
    if (rowok && l < RF::N2) rowfft_pass1_regs<N1, true>(vr, l, tile, twy);
    __syncwarp();
    cpx<double>* x = slab + (size_t)(rowok ? k : 0) * N;
    if (rowok && l < RF::N1) rowfft_pass2<N1, true>([&](int e, cpx<double> val) { x[e] = val; }, l, tile);
    __syncthreads();  // the slots are free for the next group's sweep
  }
}

// k_yz_solve with the register-resident row transforms (ny = N1 * 16): the
// CTA's rows sit unpadded in shared memory, each warp transforms RowFft::RPW
// rows at a time through its own transpose tile (twiddles from the global
// table), and the chunk scans read the lower / upper chunks' values four at a
// time.
// Otherwise the same stitched chunk solve and cluster barriers as k_yz_solve.
template <int N1, int PM>
__global__ void __launch_bounds__(512) k_yz_solve_reg(cpx<double>* __restrict__ X, const double* __restrict__ cpb,
                                                      PoissonTabs tb, const cpx<double>* __restrict__ twy, int nz,
                                                      int P) {
  using RF = RowFft<N1>;
  constexpr int ny = RF::N;
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smraw[];
  const int CS = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int kx = blockIdx.x / CS;
  const int tid = threadIdx.x, nthr = blockDim.x, nwarp = nthr >> 5;
  cpx<double>* R = reinterpret_cast<cpx<double>*>(smraw);        // P rows of ny
  cpx<double>* tiles = R + (size_t)P * ny;                          // nwarp * RPW tiles
  cpx<double>* eV = tiles + (size_t)nwarp * RF::RPW * RF::TILE;    // ny
  cpx<double>* sZ = eV + ny;                                        // ny
  double* eG = reinterpret_cast<double*>(sZ + ny);                  // ny
  double* sH = eG + ny;                                             // ny
  const int k0 = rank * P;
  const int nr = max(0, min(P, nz - k0));
  cpx<double>* slab = X + ((size_t)kx * nz + k0) * ny;
#pragma unroll 4
  for (int e = tid; e < nr * ny; e += nthr) R[e] = slab[e];
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;
  cpx<double>* tile = tiles + (size_t)(warp * RF::RPW + (sub < RF::RPW ? sub : 0)) * RF::TILE;
  auto rows_fft = [&](auto inv) {
    constexpr bool INV = decltype(inv)::value;
    for (int r0 = warp * RF::RPW; r0 < nr; r0 += nwarp * RF::RPW) {
      const int row = r0 + sub;
      const bool ok = sub < RF::RPW && row < nr;
      cpx<double>* x = R + (size_t)(ok ? row : 0) * ny;
      if (ok && l < RF::N2) rowfft_pass1<N1, INV>([&](int e) { return x[e]; }, l, tile, twy);
      __syncwarp();
      if (ok && l < RF::N1) rowfft_pass2<N1, INV>([&](int e, cpx<double> val) { x[e] = val; }, l, tile);
      __syncwarp();
    }
  };
  rows_fft(std::integral_constant<bool, false>{});
  __syncthreads();

  // one column per thread (blockDim >= ny); factors rebuilt on the fly
  const int j = tid;
  const bool colt = j < ny;
  const double K2 = colt ? tb.k2x[kx] + tb.k2y[j] : 0.0;
  double cpv[PM], gv[PM];
  cpx<double>* col = R + (colt ? j : 0);
  if (colt) {
    double cprev = cpb[((size_t)kx * CS + rank) * ny + j];
    double yr = 0.0, yi = 0.0, g = 1.0;
#pragma unroll
    for (int r = 0; r < PM; ++r) {
      if (r < nr) {
        const int k = k0 + r;
        const double cl = tb.cl[k], cr = tb.cr[k];
        const double a = (k == 0) ? 0.0 : cl;
        double bb = -(cl + cr + K2);
        if (k == 0) bb += cl;
        if (k == nz - 1) bb += cr;
        const double c = (k == nz - 1) ? 0.0 : cr;
        const double rd = 1.0 / (bb - a * cprev);
        const double cpk = (k == nz - 1) ? 0.0 : c * rd;
        const cpx<double> d = col[(size_t)r * ny];
        yr = (d.x - a * yr) * rd;
        yi = (d.y - a * yi) * rd;
        col[(size_t)r * ny] = cpx<double>{yr, yi};
        g *= -a * rd;
        gv[r] = g;
        cpv[r] = cpk;
        cprev = cpk;
      }
    }
    eV[j] = cpx<double>{yr, yi};
    eG[j] = g;
  }
  cluster.sync();
  if (colt) {
    // d'(start-1) from the lower chunks, remote reads four at a time
    double dr = 0.0, di = 0.0;
    for (int c0 = 0; c0 < rank; c0 += 4) {
      cpx<double> vv[4];
      double gg[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (c0 + q < rank) {
          vv[q] = *cluster.map_shared_rank(eV + j, c0 + q);
          gg[q] = *cluster.map_shared_rank(eG + j, c0 + q);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (c0 + q < rank) {
          dr = vv[q].x + gg[q] * dr;
          di = vv[q].y + gg[q] * di;
        }
      }
    }
    const bool gauge = (kx == 0) && (j == 0);
    double zr = 0.0, zi = 0.0, h = 1.0;
#pragma unroll
    for (int r = PM - 1; r >= 0; --r) {
      if (r < nr) {
        const int k = k0 + r;
        const cpx<double> y = col[(size_t)r * ny];
        double vr = y.x + gv[r] * dr, vi = y.y + gv[r] * di;
        if (gauge && k == nz - 1) { vr = 0.0; vi = 0.0; }
        zr = vr - cpv[r] * zr;
        zi = vi - cpv[r] * zi;
        col[(size_t)r * ny] = cpx<double>{zr, zi};
        h *= -cpv[r];
        gv[r] = h;
      }
    }
    sZ[j] = cpx<double>{zr, zi};
    sH[j] = h;
  }
  cluster.sync();
  if (colt) {
    // x(end+1) from the upper chunks, top down, remote reads four at a time
    double xr = 0.0, xi = 0.0;
    for (int c0 = CS - 1; c0 > rank; c0 -= 4) {
      cpx<double> vv[4];
      double hh[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (c0 - q > rank) {
          vv[q] = *cluster.map_shared_rank(sZ + j, c0 - q);
          hh[q] = *cluster.map_shared_rank(sH + j, c0 - q);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (c0 - q > rank) {
          xr = vv[q].x + hh[q] * xr;
          xi = vv[q].y + hh[q] * xi;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < PM; ++r) {
      if (r < nr) {
        const cpx<double> z = col[(size_t)r * ny];
        col[(size_t)r * ny] = cpx<double>{z.x + gv[r] * xr, z.y + gv[r] * xi};
      }
    }
  }
  cluster.barrier_arrive();  // this CTA reads no peer memory after here
  __syncthreads();
  rows_fft(std::integral_constant<bool, true>{});
  __syncthreads();
#pragma unroll 4
  for (int e = tid; e < nr * ny; e += nthr) slab[e] = R[e];
  cluster.barrier_wait();
}

// Inverse real FFT along x of JT rows of plane k; writes p[k][j][i] (FP64).
__global__ void __launch_bounds__(256) k_ifftx(const cpx<double>* __restrict__ X, double* __restrict__ p, int nx,
                                               int ny, int nz, FftPlan plx, const cpx<double>* __restrict__ twx,
                                               int JT) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nxh = nx / 2 + 1, rs = padded_len<double>(nx);
  cpx<double>* b0 = reinterpret_cast<cpx<double>*>(smraw);
  cpx<double>* b1 = b0 + (JT / 2) * rs;
  cpx<double>* stw = b1 + (JT / 2) * rs;  // twiddles (nx)
  const int k = blockIdx.y, j0 = blockIdx.x * JT;
  const int tid = threadIdx.x, nthr = blockDim.x;
  stage_twiddles(stw, twx, nx, tid, nthr);
  // stage the half spectra: S[r][m] in b1 (JT * nxh <= JT/2 * rs entries,
  // unpadded: this staging is not an FFT buffer)
  for (int e = tid; e < nxh * JT; e += nthr) {
    int m = e / JT, r = e - m * JT;
    cpx<double> val = X[((size_t)m * nz + k) * ny + j0 + r];
    if (m == 0 || 2 * m == nx) val.y = 0.0;  // DC / Nyquist are real (irfft ignores the imaginary part)
    b1[r * nxh + m] = val;
  }
  __syncthreads();
  for (int e = tid; e < (JT / 2) * nx; e += nthr) {
    int pr = e / nx, m = e - pr * nx;
    cpx<double> A, B;
    if (m < nxh) { A = b1[(2 * pr) * nxh + m]; B = b1[(2 * pr + 1) * nxh + m]; }
    else { A = cconj(b1[(2 * pr) * nxh + nx - m]); B = cconj(b1[(2 * pr + 1) * nxh + nx - m]); }
    b0[pr * rs + padi<double>(m)] = cmake<double>(A.x - B.y, A.y + B.x);  // A + i B
  }
  __syncthreads();
  int which = fft_rows<double, true>(b0, b1, JT / 2, rs, plx, stw, tid, nthr);
  const cpx<double>* Z = which ? b1 : b0;
  for (int e = tid; e < JT * nx; e += nthr) {
    int r = e / nx, i = e - r * nx;
    cpx<double> z = Z[(r >> 1) * rs + padi<double>(i)];
    p[pidx(k, j0 + r, i, ny, nx)] = (r & 1) ? z.y : z.x;
  }
}

}  // namespace tc
