// Kernel (e): turbulence statistics (TurbulenceStats.accumulate_statistics,
// turbstats.py:101-228) with FP64 running sums on the device.
//   profiles: per z plane, means of the cell-centred u, v, w and of the
//             fluctuation products uu, vv, ww, uw (block reductions);
//   spectra : 2-D FFTs of the fluctuation planes at k_bot / k_top (top-wall w
//             negated), |.|^2 / (nx ny)^2, walls averaged, +-kx folded.
// The six real planes travel as three complex planes (a + i b) through one
// 2-D complex FFT each and are separated afterwards.
#pragma once
#include "tc_common.cuh"
#include "tc_fft.cuh"

namespace tc {

// Cell-centred values of plane k at (j, i) (turbstats.py:114-135).
template <class T> struct CellCentre {
  const T* u; const T* v; const T* w; int nx, ny;
  const double* ubase;  // base profile of the stored u, or nullptr
  __device__ __forceinline__ double uc(int k, int j, int i) const {
    return 0.5 * ((double)u[pidx(k, j, wrap(i - 1, nx), ny, nx)] + (double)u[pidx(k, j, i, ny, nx)]) +
           (ubase ? ubase[k] : 0.0);
  }
  __device__ __forceinline__ double vc(int k, int j, int i) const {
    return 0.5 * ((double)v[pidx(k, wrap(j - 1, ny), i, ny, nx)] + (double)v[pidx(k, j, i, ny, nx)]);
  }
  __device__ __forceinline__ double wc(int k, int j, int i) const {
    return 0.5 * ((double)w[pidx(k, j, i, ny, nx)] + (double)w[pidx(k + 1, j, i, ny, nx)]);
  }
};

// One block per plane k.  prof: 5*nz running sums (U, uu, vv, ww, uw);
// means: 3*nz plane means of this sample (U, V, W) for the spectra pass.
template <class T>
__global__ void __launch_bounds__(256) k_stats_prof(const T* __restrict__ u, const T* __restrict__ v,
                                                    const T* __restrict__ w, int nx, int ny, int nz,
                                                    const double* __restrict__ ubase,
                                                    double* __restrict__ prof, double* __restrict__ means) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  CellCentre<T> C{u, v, w, nx, ny, ubase};
  const int n = nx * ny;
  double su = 0, sv = 0, sw = 0;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    int j = e / nx, i = e - j * nx;
    su += C.uc(k, j, i); sv += C.vc(k, j, i); sw += C.wc(k, j, i);
  }
  const double inv = 1.0 / (double)n;
  const double U = block_sum(su, sh) * inv;
  const double V = block_sum(sv, sh) * inv;
  const double W = block_sum(sw, sh) * inv;
  double uu = 0, vv = 0, ww = 0, uw = 0;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    int j = e / nx, i = e - j * nx;
    double a = C.uc(k, j, i) - U, b = C.vc(k, j, i) - V, c = C.wc(k, j, i) - W;
    uu += a * a; vv += b * b; ww += c * c; uw += a * c;
  }
  uu = block_sum(uu, sh) * inv;
  vv = block_sum(vv, sh) * inv;
  ww = block_sum(ww, sh) * inv;
  uw = block_sum(uw, sh) * inv;
  if (threadIdx.x == 0) {
    prof[0 * nz + k] += U; prof[1 * nz + k] += uu; prof[2 * nz + k] += vv;
    prof[3 * nz + k] += ww; prof[4 * nz + k] += uw;
    means[0 * nz + k] = U; means[1 * nz + k] = V; means[2 * nz + k] = W;
  }
}

// Pack the fluctuation planes: S0 = u_b + i w_b, S1 = u_t + i (-w_t),
// S2 = v_b + i v_t; S is [3][ny][nx] complex double.
template <class T>
__global__ void k_stats_fill(const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w, int nx,
                             int ny, int nz, int kb, int kt, const double* __restrict__ ubase,
                             const double* __restrict__ means, cpx<double>* __restrict__ S) {
  CellCentre<T> C{u, v, w, nx, ny, ubase};
  const int n = nx * ny;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    int j = e / nx, i = e - j * nx;
    double ub = C.uc(kb, j, i) - means[kb], ut = C.uc(kt, j, i) - means[kt];
    double vb = C.vc(kb, j, i) - means[nz + kb], vt = C.vc(kt, j, i) - means[nz + kt];
    double wb = C.wc(kb, j, i) - means[2 * nz + kb], wt = C.wc(kt, j, i) - means[2 * nz + kt];
    S[e] = cpx<double>{ub, wb};
    S[n + e] = cpx<double>{ut, -wt};
    S[2 * n + e] = cpx<double>{vb, vt};
  }
}

// FFT along the strided axis: CB consecutive columns (stride `cs` elements
// between successive entries of a column, `nrows` entries per column) per
// block, staged as smem rows.  Used for the y transform of the stats planes.
template <bool INV>
__global__ void __launch_bounds__(256) k_fft_cols(cpx<double>* __restrict__ S, int ncols_per_plane, int nlen,
                                                  int cs, size_t plane_stride, FftPlan pl,
                                                  const cpx<double>* __restrict__ tw, int CB) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int rs = padded_len<double>(nlen);
  cpx<double>* b0 = reinterpret_cast<cpx<double>*>(smraw);
  cpx<double>* b1 = b0 + CB * rs;
  cpx<double>* stw = b1 + CB * rs;
  stage_twiddles(stw, tw, nlen, threadIdx.x, blockDim.x);
  const int blocks_per_plane = (ncols_per_plane + CB - 1) / CB;
  const int plane = blockIdx.x / blocks_per_plane;
  const int c0 = (blockIdx.x - plane * blocks_per_plane) * CB;
  const int nc = min(CB, ncols_per_plane - c0);
  cpx<double>* base = S + plane * plane_stride + c0;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int e = tid; e < nc * nlen; e += nthr) {
    int r = e / nc, c = e - r * nc;
    b0[c * rs + padi<double>(r)] = base[(size_t)r * cs + c];
  }
  __syncthreads();
  int which = fft_rows<double, INV>(b0, b1, nc, rs, pl, stw, tid, nthr);
  const cpx<double>* Z = which ? b1 : b0;
  for (int e = tid; e < nc * nlen; e += nthr) {
    int r = e / nc, c = e - r * nc;
    base[(size_t)r * cs + c] = Z[c * rs + padi<double>(r)];
  }
}

// Contiguous-row FFT (rows of length nlen), RB rows per block.
template <bool INV>
__global__ void __launch_bounds__(256) k_fft_rows_d(cpx<double>* __restrict__ S, int nrows, int nlen, FftPlan pl,
                                                    const cpx<double>* __restrict__ tw, int RB) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int rs = padded_len<double>(nlen);
  cpx<double>* b0 = reinterpret_cast<cpx<double>*>(smraw);
  cpx<double>* b1 = b0 + RB * rs;
  cpx<double>* stw = b1 + RB * rs;
  stage_twiddles(stw, tw, nlen, threadIdx.x, blockDim.x);
  const int r0 = blockIdx.x * RB;
  const int nb = min(RB, nrows - r0);
  cpx<double>* base = S + (size_t)r0 * nlen;
  for (int e = threadIdx.x; e < nb * nlen; e += blockDim.x) {
    const int r = e / nlen, q = e - r * nlen;
    b0[r * rs + padi<double>(q)] = base[e];
  }
  __syncthreads();
  int which = fft_rows<double, INV>(b0, b1, nb, rs, pl, stw, threadIdx.x, blockDim.x);
  const cpx<double>* Z = which ? b1 : b0;
  for (int e = threadIdx.x; e < nb * nlen; e += blockDim.x) {
    const int r = e / nlen, q = e - r * nlen;
    base[e] = Z[r * rs + padi<double>(q)];
  }
}

// Separate the packed spectra and accumulate the folded, wall-averaged
// spectra (turbstats.py:176-225).  spec: 4 x (nx/2) x (ny/2), C order.
// Fold: E(kx, ky) + E(-kx, ky) = E(kx, ky) + E(kx, -ky) (real input).
__global__ void k_stats_spec(const cpx<double>* __restrict__ S, int nx, int ny, double* __restrict__ spec) {
  const int hx = nx / 2, hy = ny / 2;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= hx * hy) return;
  const int a = t / hy, b = t - a * hy;
  const int n = nx * ny;
  const double norm = 1.0 / ((double)n * (double)n);
  double Euu = 0, Evv = 0, Eww = 0, Euw = 0;
  const int kx = a + 1;
  for (int s = 0; s < 2; ++s) {
    const int ky = s == 0 ? b + 1 : ny - (b + 1);
    const int mx = (nx - kx) % nx, my = (ny - ky) % ny;
    const size_t o = (size_t)ky * nx + kx, on = (size_t)my * nx + mx;
    // pair p: A = (Z + conj Zn)/2, B = (Z - conj Zn)/(2i)
    cpx<double> F[3][2];
    for (int p = 0; p < 3; ++p) {
      cpx<double> Z = S[p * n + o], Zn = S[p * n + on];
      F[p][0] = cpx<double>{0.5 * (Z.x + Zn.x), 0.5 * (Z.y - Zn.y)};
      F[p][1] = cpx<double>{0.5 * (Z.y + Zn.y), -0.5 * (Z.x - Zn.x)};
    }
    // F[0]: (u_b, w_b), F[1]: (u_t, -w_t), F[2]: (v_b, v_t)
    auto abs2 = [](cpx<double> z) { return z.x * z.x + z.y * z.y; };
    Euu += 0.5 * (abs2(F[0][0]) + abs2(F[1][0]));
    Evv += 0.5 * (abs2(F[2][0]) + abs2(F[2][1]));
    Eww += 0.5 * (abs2(F[0][1]) + abs2(F[1][1]));
    Euw += 0.5 * ((F[0][0].x * F[0][1].x + F[0][0].y * F[0][1].y) + (F[1][0].x * F[1][1].x + F[1][0].y * F[1][1].y));
  }
  const size_t q = (size_t)a * hy + b, Q = (size_t)hx * hy;
  spec[q] += Euu * norm;
  spec[Q + q] += Evv * norm;
  spec[2 * Q + q] += Eww * norm;
  spec[3 * Q + q] += Euw * norm;
}

}  // namespace tc
