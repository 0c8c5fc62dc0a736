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
#include "tc_common.cuh"
#include "tc_fft.cuh"

namespace tc {

struct PoissonTabs {
  const double* k2x;  // nx/2+1: modified wavenumber squared (projection_fft.py:26-39)
  const double* k2y;  // ny
  const double* cl;   // nz: 1/(dz_c[k] dz_f[k])          (projection_fft.py:48)
  const double* cr;   // nz: 1/(dz_c[k+1] dz_f[k])        (projection_fft.py:49)
};

// Divergence (utils.py:226-240) of (u, v, w) scaled by `scale`, or a given
// cell field times `scale` when u == nullptr; then forward real FFT along x of
// JT rows of plane k.  Writes X[m][k][j] for m < nx/2+1.
template <class T>
__global__ void __launch_bounds__(256) k_div_fftx(Grid<T> g, const T* __restrict__ u, const T* __restrict__ v,
                                                  const T* __restrict__ w, const T* __restrict__ field,
                                                  cpx<T>* __restrict__ X, FftPlan plx,
                                                  const cpx<T>* __restrict__ twx, T scale, int JT) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxh = nx / 2 + 1;
  const int rs = nx + 2;
  cpx<T>* b0 = reinterpret_cast<cpx<T>*>(smraw);
  cpx<T>* b1 = b0 + (JT / 2) * rs;
  const int k = blockIdx.y, j0 = blockIdx.x * JT;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int e = tid; e < JT * nx; e += nthr) {
    int r = e / nx, i = e - r * nx, j = j0 + r;
    T val;
    if (u != nullptr) {
      const size_t o = pidx(k, j, i, ny, nx);
      val = (u[o] - u[pidx(k, j, wrap(i - 1, nx), ny, nx)]) * g.idx +
            (v[o] - v[pidx(k, wrap(j - 1, ny), i, ny, nx)]) * g.idy +
            (w[pidx(k + 1, j, i, ny, nx)] - w[o]) * g.idzf[k];
    } else {
      val = field[pidx(k, j, i, ny, nx)];
    }
    val *= scale;
    T* dst = reinterpret_cast<T*>(&b0[(r >> 1) * rs + i]);
    dst[r & 1] = val;
  }
  __syncthreads();
  int which = fft_rows<T, false>(b0, b1, JT / 2, rs, plx, twx, tid, nthr);
  const cpx<T>* Z = which ? b1 : b0;
  for (int e = tid; e < nxh * JT; e += nthr) {
    int m = e / JT, r = e - m * JT, pr = r >> 1;
    cpx<T> Zm = Z[pr * rs + m];
    cpx<T> Zn = cconj(Z[pr * rs + (m == 0 ? 0 : nx - m)]);
    cpx<T> out;
    if ((r & 1) == 0) out = cscale(cadd(Zm, Zn), T(0.5));
    else {
      cpx<T> d = csub(Zm, Zn);  // (Z - conj Z(-m)) / (2i) = -i/2 * d
      out = cmake<T>(T(0.5) * d.y, T(-0.5) * d.x);
    }
    X[((size_t)m * nz + k) * ny + j0 + r] = out;
  }
}

// In-place complex FFT along y of the rows X[kx][k][:] (RB rows per block).
template <class T, bool INV>
__global__ void __launch_bounds__(256) k_ffty(cpx<T>* __restrict__ X, int nrows, int ny, FftPlan ply,
                                              const cpx<T>* __restrict__ twy, int RB) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<T>* b0 = reinterpret_cast<cpx<T>*>(smraw);
  cpx<T>* b1 = b0 + RB * ny;
  const int r0 = blockIdx.x * RB;
  const int nb = min(RB, nrows - r0);
  const int tid = threadIdx.x, nthr = blockDim.x;
  cpx<T>* base = X + (size_t)r0 * ny;
  for (int e = tid; e < nb * ny; e += nthr) b0[e] = base[e];
  __syncthreads();
  int which = fft_rows<T, INV>(b0, b1, nb, ny, ply, twy, tid, nthr);
  const cpx<T>* Z = which ? b1 : b0;
  for (int e = tid; e < nb * ny; e += nthr) base[e] = Z[e];
}

// Thomas sweep along z for every mode (kx, ky), one thread per mode
// (projection_fft.py:167-215), with the tridiagonal rows of
// projection_fft.py:44-82 built on the fly.  The (0,0) mode is singular: its
// last unknown is pinned to 0 (explicit gauge) instead of dividing by the
// roundoff-level pivot.  FP64 arithmetic; d' goes to `dps` (FP64, may alias X
// when T is double), c' to shared memory.
template <class T>
__global__ void __launch_bounds__(64) k_tri(cpx<T>* __restrict__ X, cpx<double>* __restrict__ dps,
                                            PoissonTabs tb, int nxh, int ny, int nz) {
  extern __shared__ double cps[];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxh * ny) return;
  const int kx = t / ny, ky = t - kx * ny;
  const double K2 = tb.k2x[kx] + tb.k2y[ky];
  const size_t stride = ny;
  const size_t base = (size_t)kx * nz * ny + ky;
  const int bt = blockDim.x;
  double* cpl = cps + threadIdx.x;
  // forward
  double dpr = 0.0, dpi = 0.0, cprev = 0.0;
  for (int k = 0; k < nz; ++k) {
    const double cl = tb.cl[k], cr = tb.cr[k];
    double a = (k == 0) ? 0.0 : cl;
    double b = -(cl + cr + K2);
    if (k == 0) b += cl;
    if (k == nz - 1) b += cr;
    double c = (k == nz - 1) ? 0.0 : cr;
    cpx<T> dv = X[base + (size_t)k * stride];
    double den = b - a * cprev;
    double rden = 1.0 / den;
    double cpk = c * rden;
    dpr = ((double)dv.x - a * dpr) * rden;
    dpi = ((double)dv.y - a * dpi) * rden;
    cpl[(size_t)k * bt] = cpk;
    cprev = cpk;
    dps[base + (size_t)k * stride] = cpx<double>{dpr, dpi};
  }
  // backward
  double xr = dpr, xi = dpi;
  if (kx == 0 && ky == 0) { xr = 0.0; xi = 0.0; }
  X[base + (size_t)(nz - 1) * stride] = cpx<T>{(T)xr, (T)xi};
  for (int k = nz - 2; k >= 0; --k) {
    cpx<double> d = dps[base + (size_t)k * stride];
    const double cpk = cpl[(size_t)k * bt];
    xr = d.x - cpk * xr;
    xi = d.y - cpk * xi;
    X[base + (size_t)k * stride] = cpx<T>{(T)xr, (T)xi};
  }
}

// Inverse real FFT along x of JT rows of plane k; writes p[k][j][i].
template <class T>
__global__ void __launch_bounds__(256) k_ifftx(const cpx<T>* __restrict__ X, T* __restrict__ p, int nx, int ny,
                                               int nz, FftPlan plx, const cpx<T>* __restrict__ twx, int JT) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nxh = nx / 2 + 1, rs = nx + 2;
  cpx<T>* b0 = reinterpret_cast<cpx<T>*>(smraw);
  cpx<T>* b1 = b0 + (JT / 2) * rs;
  const int k = blockIdx.y, j0 = blockIdx.x * JT;
  const int tid = threadIdx.x, nthr = blockDim.x;
  // stage the half spectra: S[r][m] in b1 (JT * nxh <= JT/2 * rs entries)
  for (int e = tid; e < nxh * JT; e += nthr) {
    int m = e / JT, r = e - m * JT;
    cpx<T> val = X[((size_t)m * nz + k) * ny + j0 + r];
    if (m == 0 || 2 * m == nx) val.y = T(0);  // DC / Nyquist are real (irfft ignores the imaginary part)
    b1[r * nxh + m] = val;
  }
  __syncthreads();
  for (int e = tid; e < (JT / 2) * nx; e += nthr) {
    int pr = e / nx, m = e - pr * nx;
    cpx<T> A, B;
    if (m < nxh) { A = b1[(2 * pr) * nxh + m]; B = b1[(2 * pr + 1) * nxh + m]; }
    else { A = cconj(b1[(2 * pr) * nxh + nx - m]); B = cconj(b1[(2 * pr + 1) * nxh + nx - m]); }
    b0[pr * rs + m] = cmake<T>(A.x - B.y, A.y + B.x);  // A + i B
  }
  __syncthreads();
  int which = fft_rows<T, true>(b0, b1, JT / 2, rs, plx, twx, tid, nthr);
  const cpx<T>* Z = which ? b1 : b0;
  for (int e = tid; e < JT * nx; e += nthr) {
    int r = e / nx, i = e - r * nx;
    cpx<T> z = Z[(r >> 1) * rs + i];
    p[pidx(k, j0 + r, i, ny, nx)] = (r & 1) ? z.y : z.x;
  }
}

}  // namespace tc
