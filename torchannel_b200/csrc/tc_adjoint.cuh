// Hand-written adjoint (reverse mode) of the IMEX step, FP64.
//
// One forward IMEX step (solver.py:580-710) maps (q, r_prev, f) to
// (q', r, f') through
//   R   = nu Dxy q - A(q) + f e_u + F          (kernel a; F: optional body force)
//   q*  = q + dt (1.5 R - 0.5 r_prev)          (AB2; first step q + dt R)
//   q** = Cz^-1 Bz q*                          (CN z diffusion, kernel b)
//   q'  = P q** = q** - G L^-1 D q**           (FFT projection, kernels c, d)
//   f'  = f + (U_b - ub(q')) / dt * 0.1        (PI forcing)
//   r   = R.
// Its adjoint runs the transposes in reverse order:
//   lambda   -= (0.1 / dt) mu grad ub                       bulk / PI forcing
//   lambda** = W P W^-1 lambda                              projection
//       (P is self-adjoint in the cell / face volume inner product W:
//        <D q, phi>_Wp = -<q, G phi>_Wq on this staggered grid)
//   lambda*  = Bz^T Cz^-T lambda**                          CN (transposed rows)
//   lambda_R = c1 lambda* + lambda_r ; lambda_r <- c2 lambda*   AB2 split
//   mu      += sum_u lambda_R_u ; lambda_F += lambda_R      forcing, body force
//   lambda   = lambda* + (nu Dxy - dA[q])^T lambda_R        right-hand side
// with c1 = 1.5 dt, c2 = -0.5 dt (c1 = dt, c2 = 0 on a first step).
//
// The advection transpose is written in gather form.  Every advective flux
// is a product of two interpolants (operators.py:126-247); the fluxes sit on
// cell centres (uu, vv, ww) and on cell edges, where the same product appears
// in two components' equations (uv in adv_u's y flux and adv_v's x flux, uw in
// adv_u's z flux and adv_w's x flux, vw likewise).  A flux's adjoint is the
// difference of the adjoint right-hand sides on its two sides (divided by the
// spacing); a velocity's adjoint gathers, from the two fluxes on either side
// of it, that adjoint times the half of the other factor's interpolant.  No
// ghost term survives: w = 0 on the walls zeroes every z flux there.
// Internal layout as everywhere: [k][j][i], u/v nz planes, w nz+1 planes.
#pragma once
#include "tc_common.cuh"

namespace tc {

struct AdjRhsArgs {
  const double* u; const double* v; const double* w;      // forward state q^n
  const double* Ru; const double* Rv; const double* Rw;   // lambda_R
  double* lu; double* lv; double* lw;                     // += (nu Dxy - dA[q])^T lambda_R
  const double* idzf; const double* idzc;
  double idx, idy, nu_idx2, nu_idy2;
  int nx, ny, nz, top_neumann, rhs_fused;
};

__device__ __forceinline__ int wrp(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Gather-form transpose of the explicit right-hand side; one thread per
// (i, j, k), k in [0, nz]: u and v at cell k (k < nz), w at face k.
__global__ void __launch_bounds__(256) k_adj_rhs(AdjRhsArgs a) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= nx || j >= ny || k > nz) return;
  const size_t pl = (size_t)nx * ny;
  const double top = a.top_neumann ? 1.0 : -1.0;
  auto id = [&](int ii, int jj) { return (size_t)wrp(jj, ny) * nx + wrp(ii, nx); };
  // velocities with the z ghost rules of apply_bc_all (solver.py:50-54, 78-79)
  auto U = [&](int ii, int jj, int kk) -> double {
    if (kk < 0) return -ldg(a.u + id(ii, jj));
    if (kk >= nz) return top * ldg(a.u + (size_t)(nz - 1) * pl + id(ii, jj));
    return ldg(a.u + (size_t)kk * pl + id(ii, jj));
  };
  auto V = [&](int ii, int jj, int kk) -> double {
    if (kk < 0) return -ldg(a.v + id(ii, jj));
    if (kk >= nz) return top * ldg(a.v + (size_t)(nz - 1) * pl + id(ii, jj));
    return ldg(a.v + (size_t)kk * pl + id(ii, jj));
  };
  auto W = [&](int ii, int jj, int f) -> double {
    return (f <= 0 || f >= nz) ? 0.0 : ldg(a.w + (size_t)f * pl + id(ii, jj));
  };
  // adjoints of adv_u, adv_v, adv_w (R = ... - adv): advection is absent on
  // the edge planes i = nx-1 (u) and j = ny-1 (v) in both reference paths
  auto A = [&](int ii, int jj, int kk) -> double {
    if (kk < 0 || kk >= nz || wrp(ii, nx) == nx - 1) return 0.0;
    return -ldg(a.Ru + (size_t)kk * pl + id(ii, jj));
  };
  auto B = [&](int ii, int jj, int kk) -> double {
    if (kk < 0 || kk >= nz || wrp(jj, ny) == ny - 1) return 0.0;
    return -ldg(a.Rv + (size_t)kk * pl + id(ii, jj));
  };
  auto C = [&](int ii, int jj, int f) -> double {
    if (f <= 0 || f >= nz) return 0.0;
    return -ldg(a.Rw + (size_t)f * pl + id(ii, jj));
  };
  auto izf = [&](int kk) -> double { return (kk >= 0 && kk < nz) ? ldg(a.idzf + kk) : 0.0; };
  // flux adjoints
  auto Lxy = [&](int ii, int jj, int kk) -> double {  // uv edge (i+1/2, j+1/2) of plane kk
    return (A(ii, jj, kk) - A(ii, jj + 1, kk)) * a.idy + (B(ii, jj, kk) - B(ii + 1, jj, kk)) * a.idx;
  };
  auto Lxz = [&](int ii, int jj, int f) -> double {   // uw edge (i+1/2, face f)
    return A(ii, jj, f - 1) * izf(f - 1) - A(ii, jj, f) * izf(f) + (C(ii, jj, f) - C(ii + 1, jj, f)) * a.idx;
  };
  auto Lyz = [&](int ii, int jj, int f) -> double {   // vw edge (j+1/2, face f)
    return B(ii, jj, f - 1) * izf(f - 1) - B(ii, jj, f) * izf(f) + (C(ii, jj, f) - C(ii, jj + 1, f)) * a.idy;
  };
  const size_t o = (size_t)k * pl + (size_t)j * nx + i;
  if (k < nz) {
    // ---------------- u ----------------
    {
      auto Ux = [&](int m) { return 0.5 * (U(m - 1, j, k) + U(m, j, k)); };
      auto Cuu = [&](int m) { return (A(m - 1, j, k) - A(m, j, k)) * a.idx; };
      auto Vx = [&](int jj) { return 0.5 * (V(i, jj, k) + V(i + 1, jj, k)); };
      auto Wx = [&](int f) { return 0.5 * (W(i, j, f) + W(i + 1, j, f)); };
      double g = Ux(i) * Cuu(i) + Ux(i + 1) * Cuu(i + 1);
      g += 0.5 * (Vx(j) * Lxy(i, j, k) + Vx(j - 1) * Lxy(i, j - 1, k));
      g += 0.5 * (Wx(k + 1) * Lxz(i, j, k + 1) + Wx(k) * Lxz(i, j, k));
      auto D = [&](int ii, int jj) -> double {
        if (a.rhs_fused && wrp(ii, nx) == nx - 1) return 0.0;
        return ldg(a.Ru + (size_t)k * pl + id(ii, jj));
      };
      const double d0 = D(i, j);
      g += a.nu_idx2 * (D(i + 1, j) - 2.0 * d0 + D(i - 1, j)) + a.nu_idy2 * (D(i, j + 1) - 2.0 * d0 + D(i, j - 1));
      a.lu[o] += g;
    }
    // ---------------- v ----------------
    {
      auto Vy = [&](int m) { return 0.5 * (V(i, m - 1, k) + V(i, m, k)); };
      auto Cvv = [&](int m) { return (B(i, m - 1, k) - B(i, m, k)) * a.idy; };
      auto Uy = [&](int ii) { return 0.5 * (U(ii, j, k) + U(ii, j + 1, k)); };
      auto Wy = [&](int f) { return 0.5 * (W(i, j, f) + W(i, j + 1, f)); };
      double g = Vy(j) * Cvv(j) + Vy(j + 1) * Cvv(j + 1);
      g += 0.5 * (Uy(i) * Lxy(i, j, k) + Uy(i - 1) * Lxy(i - 1, j, k));
      g += 0.5 * (Wy(k + 1) * Lyz(i, j, k + 1) + Wy(k) * Lyz(i, j, k));
      auto D = [&](int ii, int jj) -> double {
        if (a.rhs_fused && wrp(jj, ny) == ny - 1) return 0.0;
        return ldg(a.Rv + (size_t)k * pl + id(ii, jj));
      };
      const double d0 = D(i, j);
      g += a.nu_idx2 * (D(i + 1, j) - 2.0 * d0 + D(i - 1, j)) + a.nu_idy2 * (D(i, j + 1) - 2.0 * d0 + D(i, j - 1));
      a.lv[o] += g;
    }
  }
  // ---------------- w at face k ----------------
  if (k >= 1 && k <= nz - 1) {
    const int f = k;
    auto Wz = [&](int kk) { return 0.5 * (W(i, j, kk) + W(i, j, kk + 1)); };   // cell kk
    auto Cww = [&](int kk) {                                                    // cell kk
      return C(i, j, kk) * ldg(a.idzc + kk) - C(i, j, kk + 1) * ldg(a.idzc + kk + 1);
    };
    auto Uz = [&](int ii) { return 0.5 * (U(ii, j, f - 1) + U(ii, j, f)); };
    auto Vz = [&](int jj) { return 0.5 * (V(i, jj, f - 1) + V(i, jj, f)); };
    double g = Wz(f - 1) * Cww(f - 1) + Wz(f) * Cww(f);
    g += 0.5 * (Uz(i) * Lxz(i, j, f) + Uz(i - 1) * Lxz(i - 1, j, f));
    g += 0.5 * (Vz(j) * Lyz(i, j, f) + Vz(j - 1) * Lyz(i, j - 1, f));
    auto D = [&](int ii, int jj) -> double { return ldg(a.Rw + (size_t)f * pl + id(ii, jj)); };
    const double d0 = D(i, j);
    g += a.nu_idx2 * (D(i + 1, j) - 2.0 * d0 + D(i - 1, j)) + a.nu_idy2 * (D(i, j + 1) - 2.0 * d0 + D(i, j - 1));
    a.lw[o] += g;
  }
}

// AB2 split of lambda*, body-force accumulation and the per-block sums of
// lambda_R over the u degrees of freedom (the forcing adjoint).  One thread
// per (i, j, plane k in [0, nz]); grid (ceil(nx/32), ceil(ny/8), nz+1).
struct AdjPrepArgs {
  const double* l[3];   // lambda*
  double* lr[3];        // lambda_r in, c2 lambda* out
  double* R[3];         // lambda_R out (w walls written as 0)
  double* F[3];         // += lambda_R (may be null)
  double* partials;     // one per block
  double c1, c2;
  int nx, ny, nz;
};
__global__ void __launch_bounds__(256) k_adj_prep(AdjPrepArgs a) {
  __shared__ double sh[32];
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  const size_t pl = (size_t)nx * ny;
  double su = 0.0;
  if (i < nx && j < ny) {
    const size_t o = (size_t)k * pl + (size_t)j * nx + i;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const bool dof = c < 2 ? (k < nz) : (k >= 1 && k <= nz - 1);
      if (!dof) {
        if (c == 2) a.R[2][o] = 0.0;  // walls
        continue;
      }
      const double l = a.l[c][o];
      const double r = a.c1 * l + a.lr[c][o];
      a.lr[c][o] = a.c2 * l;
      a.R[c][o] = r;
      if (a.F[c]) a.F[c][o] += r;
      if (c == 0) su = r;
    }
  }
  const double t = block_sum(su, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    a.partials[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
}

// mu += sum of the partials, in a fixed order (one block).
__global__ void __launch_bounds__(256) k_adj_mu(const double* __restrict__ partials, int n, double* mu) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int e = threadIdx.x; e < n; e += blockDim.x) s += partials[e];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *mu += s;
}

// Projection adjoint, first half: A = W^-1 (lambda - (0.1/dt) mu grad ub)
// (W = dz_f per u/v cell plane, dz_c per w face; grad ub = dx dy dz_f / V on
// u; cb = 0.1/dt * dx dy / V, or 0 with no forcing adjoint).
__global__ void __launch_bounds__(256) k_adj_scale_in(const double* lu, const double* lv, const double* lw,
                                                      double* Au, double* Av, double* Aw,
                                                      const double* __restrict__ dzf,
                                                      const double* __restrict__ dzc, const double* mu, double cb,
                                                      int nx, int ny, int nz) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  if (i >= nx || j >= ny) return;
  const size_t o = (size_t)k * nx * ny + (size_t)j * nx + i;
  const double m = mu ? *mu : 0.0;
  if (k < nz) {
    const double r = 1.0 / dzf[k];
    Au[o] = lu[o] * r - cb * m;
    Av[o] = lv[o] * r;
  }
  Aw[o] = (k >= 1 && k <= nz - 1) ? lw[o] / dzc[k] : 0.0;
}

// Projection adjoint, second half: lambda** = W (A - grad p), p the pressure
// of div A (projection.py:143-165 with dt = 1).
__global__ void __launch_bounds__(256) k_adj_project_out(const double* Au, const double* Av, const double* Aw,
                                                         const double* __restrict__ p, double* lu, double* lv,
                                                         double* lw, const double* __restrict__ dzf,
                                                         const double* __restrict__ dzc, double idx, double idy,
                                                         int nx, int ny, int nz) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  if (i >= nx || j >= ny) return;
  const size_t pl = (size_t)nx * ny;
  const size_t o = (size_t)k * pl + (size_t)j * nx + i;
  if (k < nz) {
    const double p0 = p[o];
    const double px = p[(size_t)k * pl + (size_t)j * nx + wrp(i + 1, nx)];
    const double py = p[(size_t)k * pl + (size_t)wrp(j + 1, ny) * nx + i];
    lu[o] = dzf[k] * (Au[o] - (px - p0) * idx);
    lv[o] = dzf[k] * (Av[o] - (py - p0) * idy);
  }
  if (k >= 1 && k <= nz - 1) lw[o] = dzc[k] * Aw[o] - (p[o] - p[o - pl]);
  else lw[o] = 0.0;
}

// CN adjoint tables for dt: per system (u/v: nz rows; w: nz-1 rows) the
// Thomas factors of the transposed implicit matrix C^T (sub-diagonal
// c_{m-1}, super-diagonal a_{m+1}) and the explicit CN coefficients
// (operators.py:581-644, 753-803), as k_cn_tables builds them.
// Layout per system (6 nz): aT, ivT, cpT, eA, eB, eC; tab[12 nz] = beta.
__global__ void k_adj_cn_tables(double* tab, const double* __restrict__ dzf, const double* __restrict__ dzc, int nz,
                                double nu, double dt, int top_neumann) {
  const double theta = 0.5, alpha = theta * dt * nu;
  const int sys = threadIdx.x;
  if (sys > 1) return;
  double* t = tab + (size_t)sys * 6 * nz;
  double* aT = t; double* ivT = t + nz; double* cpT = t + 2 * nz;
  double* eA = t + 3 * nz; double* eB = t + 4 * nz; double* eC = t + 5 * nz;
  const int n = sys == 0 ? nz : nz - 1;
  auto rows = [&](int m, double& am, double& bm, double& cm) {
    if (sys == 0) {
      const double dl = dzc[m], dr = dzc[m + 1], dc = dzf[m];
      const double lo = -alpha / (dl * dc), ce = 1.0 + alpha * (1.0 / dl + 1.0 / dr) / dc, up = -alpha / (dr * dc);
      am = lo; bm = ce; cm = up;
      if (m == 0) { am = 0.0; bm = ce - lo; }
      if (m == nz - 1) { bm = top_neumann ? ce + up : ce - up; cm = 0.0; }
    } else {
      const double dl = dzf[m], dr = dzf[m + 1], dcv = dzc[m + 1];
      const double lo = -alpha / (dl * dcv), ce = 1.0 + alpha * (1.0 / dl + 1.0 / dr) / dcv,
                   up = -alpha / (dr * dcv);
      am = (m == 0) ? 0.0 : lo; bm = ce; cm = (m == n - 1) ? 0.0 : up;
    }
  };
  double cpp = 0.0;
  for (int m = 0; m < n; ++m) {
    double am, bm, cm, an = 0.0, bn, cn, ap, bp, cprev = 0.0;
    rows(m, am, bm, cm);
    if (m + 1 < n) rows(m + 1, an, bn, cn);
    if (m > 0) rows(m - 1, ap, bp, cprev);
    const double sub = (m == 0) ? 0.0 : cprev;  // (C^T)_{m, m-1} = c_{m-1}
    const double sup = (m + 1 < n) ? an : 0.0;  // (C^T)_{m, m+1} = a_{m+1}
    const double rd = 1.0 / (bm - sub * cpp);
    aT[m] = sub; ivT[m] = rd; cpT[m] = sup * rd; cpp = cpT[m];
    double ea, eb, ec;
    if (sys == 0) {
      const double dl = dzc[m], dr = dzc[m + 1], dc = dzf[m];
      ea = 1.0 / (dl * dc); eb = -(1.0 / dr + 1.0 / dl) / dc; ec = 1.0 / (dr * dc);
      if (m == 0) { ea = 0.0; eb = (-1.0 / dr - 2.0 / dl) / dc; }
      if (m == nz - 1) {
        eb = top_neumann ? -1.0 / (dl * dc) : (-2.0 / dr - 1.0 / dl) / dc;
        ec = 0.0;
      }
    } else {
      const double dl = dzf[m], dr = dzf[m + 1], dcv = dzc[m + 1];
      ea = 1.0 / (dl * dcv); eb = -(1.0 / dr + 1.0 / dl) / dcv; ec = 1.0 / (dr * dcv);
      if (m == 0) ea = 0.0;
      if (m == n - 1) ec = 0.0;
    }
    eA[m] = ea; eB[m] = eb; eC[m] = ec;
  }
  if (sys == 0) tab[12 * nz] = (1.0 - theta) * dt * nu;
}

// CN adjoint, in place: y = C^-T lambda (Thomas on the transposed rows), then
// lambda* = B^T y.  u/v (comp 0, 1): row m <-> plane m, explicit stencil on
// planes m-1, m, m+1.  w (comp 2): row m <-> face m+1, explicit stencil on
// faces m-1, m, m+1 (the reference's index convention), so face g of the
// result collects y_{g-1} (its own row) and beta (cC_{g-1} y_{g-1} + cB_g y_g +
// cA_{g+1} y_{g+1}); the wall faces take nothing.  One thread per column.
// Each pass reads a column it is rewriting, so its loads are taken in blocks
// of ADJ_CN_B rows, the next block's before this block's stores (a load after
// a store to the same column would wait for it); the arithmetic is that of
// the one-row-at-a-time form.
#define ADJ_CN_B 8
__global__ void __launch_bounds__(128) k_adj_cn(double* lu, double* lv, double* lw, const double* __restrict__ tab,
                                                int nx, int ny, int nz) {
  constexpr int B = ADJ_CN_B;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int comp = blockIdx.y;
  if (col >= nx * ny) return;
  const unsigned pl = (unsigned)nx * (unsigned)ny;  // a field has fewer than 2^32 elements
  const double* t = tab + (size_t)(comp == 2 ? 1 : 0) * 6 * nz;
  const double* aT = t; const double* ivT = t + nz; const double* cpT = t + 2 * nz;
  const double* eA = t + 3 * nz; const double* eB = t + 4 * nz; const double* eC = t + 5 * nz;
  const double beta = tab[12 * nz];
  double* q = (comp == 0 ? lu : (comp == 1 ? lv : lw)) + col;
  const int n = comp < 2 ? nz : nz - 1;
  const int off = comp < 2 ? 0 : 1;  // row m lives at plane m + off
  auto row = [&](int m) -> double { return (m >= 0 && m < n) ? q[(unsigned)(m + off) * pl] : 0.0; };
  double buf[B], nxt[B];
  // forward sweep
  double yp = 0.0;
#pragma unroll
  for (int b = 0; b < B; ++b) buf[b] = row(b);
  for (int m0 = 0; m0 < n; m0 += B) {
#pragma unroll
    for (int b = 0; b < B; ++b) nxt[b] = row(m0 + B + b);
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int m = m0 + b;
      if (m < n) {
        yp = (buf[b] - aT[m] * yp) * ivT[m];
        q[(unsigned)(m + off) * pl] = yp;
      }
    }
#pragma unroll
    for (int b = 0; b < B; ++b) buf[b] = nxt[b];
  }
  // backward sweep
  double x = 0.0;
#pragma unroll
  for (int b = 0; b < B; ++b) buf[b] = row(n - 1 - b);
  for (int m1 = n - 1; m1 >= 0; m1 -= B) {
#pragma unroll
    for (int b = 0; b < B; ++b) nxt[b] = row(m1 - B - b);
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int m = m1 - b;
      if (m >= 0) {
        x = buf[b] - cpT[m] * x;
        q[(unsigned)(m + off) * pl] = x;
      }
    }
#pragma unroll
    for (int b = 0; b < B; ++b) buf[b] = nxt[b];
  }
  // explicit transpose, ascending, from a window of rows m-1, m, m+1
  if (comp < 2) {
    double ym = 0.0;
#pragma unroll
    for (int b = 0; b < B; ++b) buf[b] = row(b);
    for (int m0 = 0; m0 < n; m0 += B) {
#pragma unroll
      for (int b = 0; b < B; ++b) nxt[b] = row(m0 + B + b);
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int m = m0 + b;
        if (m < n) {
          const double y0 = buf[b], yn = (b + 1 < B) ? buf[b + 1] : nxt[0];
          double s = eB[m] * y0;
          if (m > 0) s += eC[m - 1] * ym;
          if (m + 1 < n) s += eA[m + 1] * yn;
          q[(unsigned)m * pl] = y0 + beta * s;
          ym = y0;
        }
      }
#pragma unroll
      for (int b = 0; b < B; ++b) buf[b] = nxt[b];
    }
  } else {
    // Y(m) sits at face m+1 (F(f) below, 0 past face n); output face g in
    // [1, nz-1] overwrites Y(g-1) and reads Y(g-1), Y(g), Y(g+1)
    auto F = [&](int f) -> double { return (f >= 1 && f <= n) ? q[(unsigned)f * pl] : 0.0; };
#pragma unroll
    for (int b = 0; b < B; ++b) buf[b] = F(1 + b);
    for (int g0 = 1; g0 <= nz - 1; g0 += B) {
#pragma unroll
      for (int b = 0; b < B; ++b) nxt[b] = F(g0 + B + b);
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int g = g0 + b;
        if (g <= nz - 1) {
          const double Yg1 = buf[b];
          const double Yg = (b + 1 < B) ? buf[b + 1] : nxt[b + 1 - B];
          const double Yg2 = (b + 2 < B) ? buf[b + 2] : nxt[b + 2 - B];
          double s = eC[g - 1] * Yg1;                       // row g-1 uses face g as its +1 point
          if (g <= n - 1) s += eB[g] * Yg;                  // row g uses face g as its centre
          if (g + 1 <= n - 1) s += eA[g + 1] * Yg2;         // row g+1 uses face g as its -1 point
          q[(unsigned)g * pl] = Yg1 + beta * s;
        }
      }
#pragma unroll
      for (int b = 0; b < B; ++b) buf[b] = nxt[b];
    }
  }
}

// Volume-weighted kinetic energy 0.5 sum W q^2 (W = dz_f for u, v cells,
// dz_c for w faces; the dx dy / V factor is applied by k_ke_finalize).
__global__ void __launch_bounds__(256) k_ke_partials(const double* __restrict__ u, const double* __restrict__ v,
                                                     const double* __restrict__ w, const double* __restrict__ dzf,
                                                     const double* __restrict__ dzc, double* partials, int nx,
                                                     int ny, int nz) {
  __shared__ double sh[32];
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  double s = 0.0;
  if (i < nx && j < ny) {
    const size_t o = (size_t)k * nx * ny + (size_t)j * nx + i;
    if (k < nz) s += (u[o] * u[o] + v[o] * v[o]) * dzf[k];
    if (k >= 1 && k <= nz - 1) s += w[o] * w[o] * dzc[k];
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    partials[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
}
// The forward step's adjoint hooks in one pass over the new state:
//  * (when `partials` is non-null) the block partials of the volume-weighted
//    kinetic energy 0.5 sum W q^2 as k_ke_partials forms them, skipped when
//    the weight in device memory is 0 (a captured step needs no re-capture
//    when the weight changes);
//  * (when `tape` is non-null) the copy of u, v, w into slot *ctr of the
//    state tape when *ctr < nslots (slot stride 3 (nz+1) nx ny doubles; u, v
//    with a zero top plane).
__global__ void __launch_bounds__(256) k_step_hooks(const double* __restrict__ u, const double* __restrict__ v,
                                                    const double* __restrict__ w, const double* __restrict__ dzf,
                                                    const double* __restrict__ dzc, const double* wt,
                                                    double* partials, double* tape, const int* ctr, int nslots,
                                                    int nx, int ny, int nz) {
  __shared__ double sh[32];
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  const bool in = i < nx && j < ny;
  const size_t pl = (size_t)nx * ny;
  const size_t o = (size_t)k * pl + (size_t)j * nx + i;
  if (partials) {
    double s = 0.0;
    if (*wt != 0.0 && in) {
      if (k < nz) s += (u[o] * u[o] + v[o] * v[o]) * dzf[k];
      if (k >= 1 && k <= nz - 1) s += w[o] * w[o] * dzc[k];
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0)
      partials[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
  }
  if (tape) {
    const int slot = *ctr;
    if (slot < 0 || slot >= nslots || !in) return;
    const size_t f = (size_t)(nz + 1) * pl;
    double* t = tape + (size_t)slot * 3 * f;
    t[o] = k < nz ? u[o] : 0.0;
    t[f + o] = k < nz ? v[o] : 0.0;
    t[2 * f + o] = (k >= 1 && k <= nz - 1) ? w[o] : 0.0;
  }
}
// After k_step_hooks: acc += weight coef 0.5 (sum of the partials) when
// `partials` is non-null and the weight is not 0, and the tape counter's
// advance (saturating at nslots) when `ctr` is non-null.
__global__ void __launch_bounds__(256) k_step_hooks_finalize(const double* __restrict__ partials, int n, double* acc,
                                                             const double* wt, double coef, int* ctr, int nslots) {
  __shared__ double sh[32];
  if (partials) {
    const double wv = *wt;
    if (wv != 0.0) {
      double s = 0.0;
      for (int e = threadIdx.x; e < n; e += blockDim.x) s += partials[e];
      s = block_sum(s, sh);
      if (threadIdx.x == 0) *acc += wv * coef * 0.5 * s;
    }
  }
  if (ctr && threadIdx.x == 0 && *ctr < nslots) *ctr += 1;
}

__global__ void __launch_bounds__(256) k_ke_finalize(const double* __restrict__ partials, int n, double* acc,
                                                     double coef) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int e = threadIdx.x; e < n; e += blockDim.x) s += partials[e];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) *acc += coef * 0.5 * s;
}
// lambda += coef W q  (the gradient of coef * 0.5 sum W q^2).
__global__ void __launch_bounds__(256) k_ke_seed(const double* __restrict__ u, const double* __restrict__ v,
                                                 const double* __restrict__ w, double* lu, double* lv, double* lw,
                                                 const double* __restrict__ dzf, const double* __restrict__ dzc,
                                                 double coef, int nx, int ny, int nz) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  if (i >= nx || j >= ny) return;
  const size_t o = (size_t)k * nx * ny + (size_t)j * nx + i;
  if (k < nz) {
    lu[o] += coef * dzf[k] * u[o];
    lv[o] += coef * dzf[k] * v[o];
  }
  if (k >= 1 && k <= nz - 1) lw[o] += coef * dzc[k] * w[o];
}

// Body force of the forward step: q* += cq F, r += cr F (cr = 0 without a
// stored history), over the degrees of freedom.
__global__ void __launch_bounds__(256) k_add_body(double* us, double* vs, double* ws, double* ru, double* rv,
                                                  double* rw, const double* __restrict__ fu,
                                                  const double* __restrict__ fv, const double* __restrict__ fw,
                                                  double cq, double cr, int nx, int ny, int nz) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  if (i >= nx || j >= ny) return;
  const size_t o = (size_t)k * nx * ny + (size_t)j * nx + i;
  if (k < nz) {
    us[o] += cq * fu[o];
    vs[o] += cq * fv[o];
    if (cr != 0.0) { ru[o] += cr * fu[o]; rv[o] += cr * fv[o]; }
  }
  if (k >= 1 && k <= nz - 1) {
    ws[o] += cq * fw[o];
    if (cr != 0.0) rw[o] += cr * fw[o];
  }
}

}  // namespace tc
