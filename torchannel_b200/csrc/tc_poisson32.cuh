// Single-precision Poisson middle (mixed precision, optional): for one kx
// slab of the FP32 spectrum X[kx][k][:] per CTA,
//   [FFT along y] -> [Thomas along z per ky] -> [inverse FFT along y]
// (projection_fft.py:117-139 and :167-215) with the whole slab resident in
// shared memory, so that the spectrum crosses HBM once in and once out and
// no intermediate pass touches it.
//
// * The slab arrives by bulk copies of the tensor memory accelerator
//   (cp.async.bulk, one per chunk of rows, each completing on its own
//   mbarrier), so that the y transforms of the first rows start while the
//   later rows are still in flight.
// * Row transforms: the register split N = N1 N2 of tc_fft_reg.cuh in FP32,
//   done in place in the row's own shared memory (the transpose tile is the
//   row itself, its entries rotated by k1 so that neither pass has bank
//   conflicts); the inverse writes its output rows straight to HBM.
// * z solve: one thread per (ky, real / imaginary part) sweeps the column in
//   shared memory with the per-mode LU factors of k_tri_factors, rounded to
//   FP32 once; the factor loads run two blocks of levels ahead of the
//   recurrence.  The (0,0) mode and the lowest wavenumbers (kx < 3 and
//   |ky| < 3) are solved in FP64 with the FP64 factors (the (0,0) mode
//   gauged as in k_tri_lu: x_{nz-1} = 0).
//
// The step that uses it solves for the increment of p over a base pressure
// p_b (the previous step's p): right-hand side div(u**)/dt - L p_b
// (k_base_lap), projection with the gradient of p_b + dp summed in FP64.  FP32
// rounding then scales with the change of p over a step, not with p, whose
// own FP32 rounding would reach the post-projection divergence amplified by
// dt / (dz_c dz_f) next to the walls.
#pragma once
#include "tc_async.cuh"
#include "tc_common.cuh"
#include "tc_fft_reg.cuh"

namespace tc {

#define YZ32_CHUNKS 8          // bulk copies (and barriers) per slab
#define YZ32_WAIT_LIMIT (1u << 21)
#define YZ32_B 16              // levels per factor-load block of the FP32 z sweeps
#define YZ32_B64 16            // ... of the FP64 (low-mode) sweeps
#define YZ32_NLOW 3            // FP64 modes: kx < 3 and ky < 3 or ky > ny - 3

// Threads of k_yz32 for ny = 16 K: one per (ky, part) of the z solve, at
// least 8 warps.
template <int K> __host__ __device__ constexpr int yz32_threads() {
  return 2 * 16 * K < 256 ? 256 : (2 * 16 * K + 31) / 32 * 32;
}

// FP64 d' columns of the low modes of one kx slab: (2 YZ32_NLOW - 1) ky
// values x 2 parts x nz levels.
__host__ __device__ inline size_t yz32_low_doubles(int nz) { return (size_t)(2 * YZ32_NLOW - 1) * 2 * nz; }

// Shared memory of k_yz32 for ny = N and nz levels: the slab, the FP32
// twiddles, a_k in FP32 (even count), the barriers and the low modes' FP64
// d' columns.
__host__ __device__ inline size_t yz32_smem_bytes(int N, int nz) {
  return (size_t)nz * N * 8 + (size_t)N * 8 + (size_t)((nz + 1) & ~1) * 4 + YZ32_CHUNKS * 8 +
         yz32_low_doubles(nz) * 8;
}

// One row of N = N1 N2 FP32 complex values in shared memory, transformed in
// place (forward: natural order left in `row`; `st(e, value)` receives
// element e of the result in either direction, after every lane has read
// its inputs).  All lanes of the warp call it; `ok` marks lanes with a row,
// `l` is the lane within the row's lane group.
template <int K, bool INV, class ST>
__device__ __forceinline__ void row32_fft(cpx<float>* row, int l, bool ok, const cpx<float>* tw, ST st) {
  using RF = RowFft<K>;
  constexpr int N1 = RF::N1, N2 = RF::N2;
  cpx<float> v[N1];
  const bool p1 = ok && l < N2;
  if (p1) {
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = row[N2 * n1 + l];
    Dft<N1, INV, float>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
      cpx<float> w = tw[l * k1];
      if (INV) w.y = -w.y;
      v[k1] = cmul(v[k1], w);
    }
  }
  __syncwarp();
  // transpose tile (k1, n2) at row[k1 N2 + (n2 + k1) mod N2]
  if (p1) {
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) row[k1 * N2 + ((l + k1) & (N2 - 1))] = v[k1];
  }
  __syncwarp();
  const bool p2 = ok && l < N1;
  cpx<float> b[N2];
  if (p2) {
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) b[n2] = row[l * N2 + ((n2 + l) & (N2 - 1))];
    Dft<N2, INV, float>::run(b);
  }
  __syncwarp();
  if (p2) {
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) st(l + N1 * k2, b[k2]);
  }
  __syncwarp();
}

// Thomas sweeps of one column part: forward d'_k = (d_k - a_k d'_{k-1})
// rden_k from the FP32 column `col` (levels `stride` floats apart) into
// `dq` (levels `dqs` apart: the column itself for FP32 arithmetic, an FP64
// scratch column for the FP64 modes), backward x_k = d'_k - c'_k x_{k+1}
// (x_{nz-1} = d'_{nz-1}, or 0 when gauged) into `col`.  R: arithmetic type
// of the recurrences, the factor tables ([k] at stride `ts`) and a_k.
template <class R, int B>
__device__ __forceinline__ void yz32_sweep(float* col, int stride, R* dq, int dqs, const R* __restrict__ rd,
                                           const R* __restrict__ cpt, const R* a_tab, int ts, int nz, bool gauge) {
  R fa[B], fb[B];
  auto load = [&](R (&f)[B], const R* __restrict__ tab, int k0, int dir) {
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int k = k0 + dir * b;
      f[b] = (k >= 0 && k < nz) ? ldg(tab + (size_t)k * ts) : (R)0;
    }
  };
  R dp = (R)0;
  auto up = [&](const R (&f)[B], int k0) {
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int k = k0 + b;
      if (k < nz) {
        const R a = (k == 0) ? (R)0 : a_tab[k];
        const R d = (R)col[(size_t)k * stride];
        dp = fma(-(a * f[b]), dp, d * f[b]);
        dq[(size_t)k * dqs] = dp;
      }
    }
  };
  load(fa, rd, 0, 1);
  for (int k0 = 0; k0 < nz; k0 += 2 * B) {
    load(fb, rd, k0 + B, 1);
    up(fa, k0);
    load(fa, rd, k0 + 2 * B, 1);
    up(fb, k0 + B);
  }
  // the backward sweep starts from x_{nz-1} = d'_{nz-1} (the singular (0,0)
  // mode: 0)
  R x = gauge ? (R)0 : dp;
  col[(size_t)(nz - 1) * stride] = (float)x;
  auto dn = [&](const R (&f)[B], int k1) {
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int k = k1 - b;
      if (k >= 0) {
        x = dq[(size_t)k * dqs] - f[b] * x;
        col[(size_t)k * stride] = (float)x;
      }
    }
  };
  load(fa, cpt, nz - 2, -1);
  for (int k1 = nz - 2; k1 >= 0; k1 -= 2 * B) {
    load(fb, cpt, k1 - B, -1);
    dn(fa, k1);
    load(fa, cpt, k1 - 2 * B, -1);
    dn(fb, k1 - B);
  }
}

// One CTA per kx slab (gridDim.x = nx/2+1), ny = RowFft<K>::N, blockDim.x a
// multiple of 32 and >= 2 ny; `err` gets TCE_TIMEOUT if a bulk copy did not
// complete within the wait limit (the CTA then waits, bounded, for its copies
// and returns without computing).
template <int K>
__global__ void __launch_bounds__(yz32_threads<K>()) k_yz32(cpx<float>* __restrict__ X, const float* __restrict__ rden32,
                                               const float* __restrict__ cp32, const double* __restrict__ rden64,
                                               const double* __restrict__ cp64, const double* __restrict__ cl,
                                               const cpx<float>* __restrict__ tw32, int nz,
                                               int* __restrict__ err) {
  using RF = RowFft<K>;
  constexpr int N = RF::N;
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<float>* slab = reinterpret_cast<cpx<float>*>(smraw);        // nz rows of N
  cpx<float>* stw = slab + (size_t)nz * N;                         // N twiddles
  float* scl = reinterpret_cast<float*>(stw + N);                  // a_k = cl[k] in FP32
  uint64_t* bar = reinterpret_cast<uint64_t*>(scl + ((nz + 1) & ~1));
  double* dlow = reinterpret_cast<double*>(bar + YZ32_CHUNKS);     // low modes' d' columns
  const int kx = blockIdx.x;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int rc = (nz + YZ32_CHUNKS - 1) / YZ32_CHUNKS;            // rows per chunk
  const int nch = (nz + rc - 1) / rc;                              // chunks with rows
  cpx<float>* gslab = X + (size_t)kx * nz * N;
  if (tid == 0) {
    for (int c = 0; c < nch; ++c) mbar_init(&bar[c], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (tid == 0) {
    for (int c = 0; c < nch; ++c) {
      const int r0 = c * rc, nr = min(rc, nz - r0);
      const unsigned bytes = (unsigned)nr * N * (unsigned)sizeof(cpx<float>);
      mbar_expect_tx(&bar[c], bytes);
      bulk_load(slab + (size_t)r0 * N, gslab + (size_t)r0 * N, bytes, &bar[c]);
    }
  }
  for (int e = tid; e < N; e += nthr) stw[e] = tw32[e];
  for (int e = tid; e < nz; e += nthr) scl[e] = (float)cl[e];
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, nwarp = nthr >> 5;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;
  bool waited = true;
  // forward transforms along y, each warp's rows once their chunk is in
  for (int r0 = warp * RF::RPW; r0 < nz; r0 += nwarp * RF::RPW) {
    const int c0 = r0 / rc, c1 = min(r0 + RF::RPW - 1, nz - 1) / rc;
    for (int c = c0; c <= c1; ++c) waited = waited && mbar_wait_bounded(&bar[c], 0, YZ32_WAIT_LIMIT);
    const int r = r0 + sub;
    const bool ok = waited && sub < RF::RPW && r < nz;
    cpx<float>* row = slab + (size_t)(ok ? r : 0) * N;
    row32_fft<K, false>(row, l, ok, stw, [&](int e, cpx<float> val) { row[e] = val; });
  }
  if (__syncthreads_or(!waited)) {
    if (tid == 0) {
      for (int c = 0; c < nch; ++c) mbar_wait_bounded(&bar[c], 0, YZ32_WAIT_LIMIT);
      atomicOr(err, TCE_TIMEOUT);
    }
    return;
  }
  // z solve: thread (ky, part)
  for (int t = tid; t < 2 * N; t += nthr) {
    const int ky = t >> 1, part = t & 1;
    float* col = reinterpret_cast<float*>(slab) + 2 * ky + part;
    const size_t tb = (size_t)kx * nz * N + ky;
    const bool gauge = kx == 0 && ky == 0;
    constexpr int nlow = YZ32_NLOW;
    if (kx < nlow && (ky < nlow || ky > N - nlow)) {
      const int q = ky < nlow ? ky : ky - (N - 2 * nlow + 1);
      double* dq = dlow + ((size_t)q * 2 + part) * nz;
      yz32_sweep<double, YZ32_B64>(col, 2 * N, dq, 1, rden64 + tb, cp64 + tb, cl, N, nz, gauge);
    } else {
      yz32_sweep<float, YZ32_B>(col, 2 * N, col, 2 * N, rden32 + tb, cp32 + tb, scl, N, nz, gauge);
    }
  }
  __syncthreads();
  // inverse transforms along y, results straight to HBM
  for (int r0 = warp * RF::RPW; r0 < nz; r0 += nwarp * RF::RPW) {
    const int r = r0 + sub;
    const bool ok = sub < RF::RPW && r < nz;
    cpx<float>* row = slab + (size_t)(ok ? r : 0) * N;
    cpx<float>* grow = gslab + (size_t)(ok ? r : 0) * N;
    row32_fft<K, true>(row, l, ok, stw, [&](int e, cpx<float> val) { grow[e] = val; });
  }
}

// L p_b of the base pressure (FP32 in, FP64 arithmetic, FP32 out): 3-point
// periodic differences in x and y and the z rows of projection_fft.py:44-82
// with their Neumann closures, the operator the solve inverts.
__global__ void __launch_bounds__(256) k_base_lap(const float* __restrict__ p, float* __restrict__ lp, int nx, int ny,
                                                  int nz, double idx2, double idy2, const double* __restrict__ cl,
                                                  const double* __restrict__ cr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
  if (i >= nx || j >= ny) return;
  const size_t o = pidx(k, j, i, ny, nx);
  const double c = (double)p[o];
  const double xm = (double)p[pidx(k, j, i == 0 ? nx - 1 : i - 1, ny, nx)];
  const double xp = (double)p[pidx(k, j, i == nx - 1 ? 0 : i + 1, ny, nx)];
  const double ym = (double)p[pidx(k, j == 0 ? ny - 1 : j - 1, i, ny, nx)];
  const double yp = (double)p[pidx(k, j == ny - 1 ? 0 : j + 1, i, ny, nx)];
  double l = (xp - 2.0 * c + xm) * idx2 + (yp - 2.0 * c + ym) * idy2;
  if (k < nz - 1) l += cr[k] * ((double)p[o + (size_t)nx * ny] - c);
  if (k > 0) l -= cl[k] * (c - (double)p[o - (size_t)nx * ny]);
  lp[o] = (float)l;
}

// FP32 copies of the per-mode factor tables (k_tri_factors) for the
// single-precision sweeps.
__global__ void k_tri_factors32(const double* __restrict__ rden, const double* __restrict__ cp,
                                float* __restrict__ rden32, float* __restrict__ cp32, size_t n) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    rden32[e] = (float)rden[e];
    cp32[e] = (float)cp[e];
  }
}

}  // namespace tc
