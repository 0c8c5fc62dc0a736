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
