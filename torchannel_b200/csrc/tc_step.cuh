// Time-step kernels: explicit RHS + AB2 update (kernel a), Crank-Nicolson
// z-diffusion (kernel b), projection + bulk sum + PI forcing (kernel d), CFL
// and diagnostics reductions, and reference-layout conversions.
#pragma once
#include "tc_common.cuh"
#undef TC_FILE_ID
#define TC_FILE_ID 1

namespace tc {

// ---------------------------------------------------------------------------
// Field accessors (see the layout note in tc_common.cuh)
// ---------------------------------------------------------------------------
template <class T> struct Acc {
  const T* __restrict__ q;
  int nx, ny, nz;
  T top;  // sign of the top-wall ghost of u/v: -1 no-slip, +1 free-slip
  const T* __restrict__ base;  // per-plane base profile added to the stored values, or nullptr
  __device__ __forceinline__ T b(int k) const { return base ? ldg(base + k) : T(0); }
  // cell-centred u/v plane k in [-1, nz] (total value: stored + base)
  __device__ __forceinline__ T c(int k, int j, int i) const {
    if (k < 0) return -(ldg(q + pidx(0, j, i, ny, nx)) + b(0));
    if (k >= nz) return top * (ldg(q + pidx(nz - 1, j, i, ny, nx)) + b(nz - 1));
    return ldg(q + pidx(k, j, i, ny, nx)) + b(k);
  }
  // w face f in [0, nz] (walls stored as zeros)
  __device__ __forceinline__ T f(int k, int j, int i) const { return ldg(q + pidx(k, j, i, ny, nx)); }
};

template <class T> __device__ __forceinline__ T sq(T a) { return a * a; }

// Scheme of the explicit update.
enum : int {
  UPD_AB2 = 0,     // r = rhs + forcing; q* = q + dt(1.5 r - 0.5 r_prev) (Euler without history)
  UPD_FE = 1,      // q* = q + dt rhs; u gets + dt * 1.0 (solver.py:552-554)
  UPD_RHS_ONLY = 2 // write rhs (no forcing) to r and stop (operator-level hook)
};

// ---------------------------------------------------------------------------
// Kernel (a): fused staggered advection + explicit diffusion + forcing + AB2.
//
// Reference: advection_u/v/w (operators.py:126-247), diffusion_xy_u/v/w
// (:474-548), diffusion_u/v/w (:18-124), compute_momentum_rhs_fused_imex
// (:1037-1225) and _v2 (:818-1034), AB2 combine solver.py:626-651.
// FULL=false: IMEX (x/y diffusion only); FULL=true: full Laplacian (AB2/FE).
//
// A block owns a RHS_TX x RHS_TY (rhs_ty<T>()) tile and RHS_KB (rhs_kb<T>())
// consecutive planes k = kb..kb+RHS_KB-1 (u, v at cell k, w at face k).  It
// first stages the u, v, w planes kb-1 .. kb+RHS_KB with a one-cell periodic
// halo (z ghosts applied) in shared memory -- every load of the block is
// independent and issued up front; halo offsets are computed once per thread
// -- then evaluates the stencils up its columns from shared memory
// (rhs_stencils).  Edge planes: internal i = nx-1 is reference u[nx] and
// j = ny-1 is v[:, ny]; both reference paths omit advection there, the
// separate-op path keeps the diffusion, the fused path writes 0
// (operators.py:1122,1173).
// ---------------------------------------------------------------------------
#define RHS_TX 32
// tile rows and planes per block: 8 x 4 in FP32, 8 x 3 in FP64 (static
// shared memory <= 48 KB)
template <class T> __host__ __device__ constexpr int rhs_ty() { return 8; }
template <class T> __host__ __device__ constexpr int rhs_kb() { return sizeof(T) == 8 ? 3 : 4; }
#define RHS_HX (RHS_TX + 2)

// Arithmetic with explicit rounding for the stencils below: every kernel
// that evaluates them (one tile per block, tensor-copy staging, the ensemble
// loops) produces the same bits, whatever the compiler would contract.
template <class T> struct Rn;
template <> struct Rn<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
};
template <> struct Rn<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
};

// The stencils of one thread's column of KB planes k = kb .. kb+KB-1 (u, v at
// cell k, w at face k), marching up in z over a staged tile: slot s of the
// shared arrays holds plane kb-1+s (slots 0 .. KB+1), (cy, cx) is the thread's
// point.  The tile holds the stored values (u - U0[k] in mixed precision; z
// ghosts with their sign rule applied); U0 enters the sums of u analytically.
//
// Each flux of the staggered advection is formed once per point and plane:
//  * uu at i +- 1/2 and vv at j +- 1/2 (cell centres),
//  * uv at the corners (i+1/2, j+1/2) (for u and v), (i+1/2, j-1/2) (u),
//    (i-1/2, j+1/2) (v),
//  * uw at (i +- 1/2, face k+1), vw at (j +- 1/2, face k+1) and ww at cell k:
//    formed with plane k+1 and carried to the next plane, where the face is
//    face k (u's and v's lower flux, w's four side fluxes, ww below).
// With the plane values that the next plane needs also carried in registers,
// a plane costs 17 shared loads (6 of u, 6 of v, 5 of w).  A flux is the
// product of two unscaled sums; the factors 0.5 of both interpolations are
// folded into the difference quotient as 0.25 / delta (exact: powers of two).
// The fluxes of face kb are formed before the first plane by the same
// expressions, so the results do not depend on KB or on the tile shape.
// Per-tile constants of the march (FP32 storage): U0 of slot s with the
// z-ghost rule's sign (KB + 2 values), then 1/dz_f[k] and 1/dz_c[k] of the
// tile's planes k = kb .. kb+KB-1 (KB each; 0 beyond the grid).  Entry e of
// the table, so that a kernel can stage it in shared memory before its tile
// lands and the march reads it there instead of waiting on global loads.
template <class T, int KB> __host__ __device__ constexpr int rhs_pre_count() { return 3 * KB + 2; }
template <class T, int KB>
__device__ __forceinline__ T rhs_pre_value(const Grid<T>& g, int kb, int e) {
  const int nz = g.nz;
  if (e < KB + 2) {
    const int p = kb - 1 + e;
    if (sizeof(T) != 4 || !g.ubase_t) return T(0);
    const int pc = p < 0 ? 0 : (p >= nz ? nz - 1 : p);
    const T sgn = p < 0 ? T(-1) : (p >= nz ? (g.top_neumann ? T(1) : T(-1)) : T(1));
    return TC_IN(pc, nz, 1) ? sgn * ldg(g.ubase_t + pc) : T(0);
  }
  const int k = kb + (e < 2 * KB + 2 ? e - (KB + 2) : e - (2 * KB + 2));
  if (k >= nz) return T(0);
  return e < 2 * KB + 2 ? (TC_IN(k, nz, 1) ? ldg(g.idzf + k) : T(0)) : (TC_IN(k, nz + 1, 1) ? ldg(g.idzc + k) : T(0));
}

// pre: the table of rhs_pre_value in shared memory, or nullptr (the march
// loads the constants itself).
template <class T, bool FULL, int UPD, int KB, int HY, int HX>
__device__ __forceinline__ void rhs_march(const Grid<T>& g, const T (*__restrict__ su)[HY][HX],
                                          const T (*__restrict__ sv)[HY][HX], const T (*__restrict__ sw)[HY][HX],
                                          int cx, int cy, int i, int j, bool active, int kb, T* __restrict__ us,
                                          T* __restrict__ vs, T* __restrict__ ws, T* __restrict__ ru,
                                          T* __restrict__ rv, T* __restrict__ rw, T (&hru)[KB], T (&hrv)[KB],
                                          T (&hrw)[KB], T forcing, T dt, int have_hist,
                                          const T* __restrict__ pre = nullptr) {
  using R = Rn<T>;
  constexpr bool HB = sizeof(T) == 4;  // mixed precision: u stored as u - U0[k]
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t plane = (size_t)nx * ny;
  const size_t ncell = plane * nz, nface = plane * (nz + 1);  // field extents (bounds-checked builds)
  (void)ncell; (void)nface;
  // U0 of slot s (plane kb-1+s) with the z-ghost rule's sign
  T bs[KB + 2];
#pragma unroll
  for (int s = 0; s < KB + 2; ++s) bs[s] = pre ? pre[s] : rhs_pre_value<T, KB>(g, kb, s);
  const T qx = T(0.25) * g.idx, qy = T(0.25) * g.idy;
  const bool edge_u = (i == nx - 1), edge_v = (j == ny - 1);
  // plane kb-1 (slot 0) and plane kb (slot 1)
  T pU0 = su[0][cy][cx], pV0 = sv[0][cy][cx], pW0 = sw[0][cy][cx];
  T cU0 = su[1][cy][cx], cUxm = su[1][cy][cx - 1], cV0 = sv[1][cy][cx], cVym = sv[1][cy - 1][cx];
  T cW0 = sw[1][cy][cx], cWxm = sw[1][cy][cx - 1], cWxp = sw[1][cy][cx + 1];
  T cWym = sw[1][cy - 1][cx], cWyp = sw[1][cy + 1][cx];
  // fluxes of face kb
  T Fuw_p, Fuw_m, Fvw_p, Fvw_m, Fww;
  {
    const T bz = HB ? R::add(bs[0], bs[1]) : T(0);
    T su_p = R::add(pU0, cU0), su_m = R::add(su[0][cy][cx - 1], cUxm);
    if (HB) { su_p = R::add(su_p, bz); su_m = R::add(su_m, bz); }
    Fuw_p = R::mul(R::add(cW0, cWxp), su_p);
    Fuw_m = R::mul(R::add(cWxm, cW0), su_m);
    Fvw_p = R::mul(R::add(cW0, cWyp), R::add(pV0, cV0));
    Fvw_m = R::mul(R::add(cWym, cW0), R::add(sv[0][cy - 1][cx], cVym));
    const T sww = R::add(pW0, cW0);
    Fww = R::mul(sww, sww);
  }
  // 32-bit offsets: a field has fewer than 2^32 elements (tc_create refuses
  // larger grids), so one wide multiply-add forms each store address
  unsigned o = (unsigned)kb * (unsigned)plane + (unsigned)j * (unsigned)nx + (unsigned)i;
#pragma unroll
  for (int kk = 0; kk < KB; ++kk, o += (unsigned)plane) {
    const int k = kb + kk;
    if (k >= nz) break;
    const int s0 = kk + 1, sp = kk + 2;
    // plane k: the in-plane neighbours not carried
    const T Uxp = su[s0][cy][cx + 1], Uym = su[s0][cy - 1][cx], Uyp = su[s0][cy + 1][cx];
    const T Uypm = su[s0][cy + 1][cx - 1];
    const T Vxm = sv[s0][cy][cx - 1], Vxp = sv[s0][cy][cx + 1], Vyp = sv[s0][cy + 1][cx];
    const T Vymp = sv[s0][cy - 1][cx + 1];
    // plane k+1
    const T nU0 = su[sp][cy][cx], nUxm = su[sp][cy][cx - 1], nV0 = sv[sp][cy][cx], nVym = sv[sp][cy - 1][cx];
    const T nW0 = sw[sp][cy][cx], nWxm = sw[sp][cy][cx - 1], nWxp = sw[sp][cy][cx + 1];
    const T nWym = sw[sp][cy - 1][cx], nWyp = sw[sp][cy + 1][cx];
    const T b2 = HB ? R::add(bs[s0], bs[s0]) : T(0);
    const T bz = HB ? R::add(bs[s0], bs[sp]) : T(0);
    auto ub = [&](T s, T b) { return HB ? R::add(s, b) : s; };
    // fluxes of plane k
    const T Sa = ub(R::add(cU0, Uxp), b2), Sb = ub(R::add(cUxm, cU0), b2);
    const T Fuu = R::fma(Sa, Sa, -R::mul(Sb, Sb));
    const T Sc = R::add(cV0, Vyp), Sd = R::add(cVym, cV0);
    const T Fvv = R::fma(Sc, Sc, -R::mul(Sd, Sd));
    const T Fuv_pp = R::mul(R::add(cV0, Vxp), ub(R::add(cU0, Uyp), b2));
    const T Fuv_pm = R::mul(R::add(cVym, Vymp), ub(R::add(Uym, cU0), b2));
    const T Fuv_mp = R::mul(ub(R::add(cUxm, Uypm), b2), R::add(Vxm, cV0));
    // fluxes of face k+1 (carried)
    const T Fuw_p1 = R::mul(R::add(nW0, nWxp), ub(R::add(cU0, nU0), bz));
    const T Fuw_m1 = R::mul(R::add(nWxm, nW0), ub(R::add(cUxm, nUxm), bz));
    const T Fvw_p1 = R::mul(R::add(nW0, nWyp), R::add(cV0, nV0));
    const T Fvw_m1 = R::mul(R::add(nWym, nW0), R::add(cVym, nVym));
    const T sww = R::add(cW0, nW0);
    const T Fww1 = R::mul(sww, sww);
    if (active) {
      const T idzf = pre ? pre[KB + 2 + kk] : g.idzf[k];
      const T qzf = T(0.25) * idzf;
      // ---------------- u at cell k ----------------
      {
        T r = T(0);
        if (!(edge_u && g.rhs_fused)) {
          const T lx = R::add(R::fma(T(-2), cU0, Uxp), cUxm), ly = R::add(R::fma(T(-2), cU0, Uyp), Uym);
          r = R::fma(g.nu_idx2, lx, R::mul(g.nu_idy2, ly));
          if (FULL) {
            T dp = R::sub(nU0, cU0), dm = R::sub(cU0, pU0);
            if (HB) { dp = R::add(dp, R::sub(bs[sp], bs[s0])); dm = R::add(dm, R::sub(bs[s0], bs[kk])); }
            const T t = R::sub(R::mul(dp, g.idzc[k + 1]), R::mul(dm, g.idzc[k]));
            r = R::fma(R::mul(g.nu, idzf), t, r);
          }
        }
        if (!edge_u) r = R::sub(r, R::fma(R::sub(Fuw_p1, Fuw_p), qzf, R::fma(R::sub(Fuv_pp, Fuv_pm), qy, R::mul(Fuu, qx))));
        if (UPD == UPD_RHS_ONLY) {
          if (TC_IN(o, ncell, 1)) ru[o] = r;
        } else if (UPD == UPD_FE) {
          if (TC_IN(o, ncell, 1)) us[o] = R::add(R::fma(dt, r, cU0), dt);
        } else {
          r = R::add(r, forcing);
          const T a = have_hist ? R::fma(T(1.5), r, R::mul(T(-0.5), hru[kk])) : r;
          if (TC_IN(o, ncell, 1)) us[o] = R::fma(dt, a, cU0);
          if (TC_IN(o, ncell, 1)) ru[o] = r;
        }
      }
      // ---------------- v at cell k ----------------
      {
        T r = T(0);
        if (!(edge_v && g.rhs_fused)) {
          const T lx = R::add(R::fma(T(-2), cV0, Vxp), Vxm), ly = R::add(R::fma(T(-2), cV0, Vyp), cVym);
          r = R::fma(g.nu_idx2, lx, R::mul(g.nu_idy2, ly));
          if (FULL) {
            const T t = R::sub(R::mul(R::sub(nV0, cV0), g.idzc[k + 1]), R::mul(R::sub(cV0, pV0), g.idzc[k]));
            r = R::fma(R::mul(g.nu, idzf), t, r);
          }
        }
        if (!edge_v) r = R::sub(r, R::fma(R::sub(Fvw_p1, Fvw_p), qzf, R::fma(R::sub(Fuv_pp, Fuv_mp), qx, R::mul(Fvv, qy))));
        if (UPD == UPD_RHS_ONLY) {
          if (TC_IN(o, ncell, 1)) rv[o] = r;
        } else if (UPD == UPD_FE) {
          if (TC_IN(o, ncell, 1)) vs[o] = R::fma(dt, r, cV0);
        } else {
          const T a = have_hist ? R::fma(T(1.5), r, R::mul(T(-0.5), hrv[kk])) : r;
          if (TC_IN(o, ncell, 1)) vs[o] = R::fma(dt, a, cV0);
          if (TC_IN(o, ncell, 1)) rv[o] = r;
        }
      }
      // ---------------- w at face k ----------------
      if (k >= 1) {
        const T lx = R::add(R::fma(T(-2), cW0, cWxp), cWxm), ly = R::add(R::fma(T(-2), cW0, cWyp), cWym);
        T r = R::fma(g.nu_idx2, lx, R::mul(g.nu_idy2, ly));
        // z term of diffusion_w divides by dz_c[K-1] (operators.py:120,1025)
        if (FULL) {
          const T t = R::sub(R::mul(R::sub(nW0, cW0), g.idzf[k]), R::mul(R::sub(cW0, pW0), g.idzf[k - 1]));
          r = R::fma(R::mul(g.nu, g.idzc[k - 1]), t, r);
        }
        const T dww = R::mul(R::sub(Fww1, Fww), T(0.25) * (pre ? pre[2 * KB + 2 + kk] : g.idzc[k]));
        r = R::sub(r, R::fma(R::sub(Fuw_p, Fuw_m), qx, R::fma(R::sub(Fvw_p, Fvw_m), qy, dww)));
        if (UPD == UPD_RHS_ONLY) {
          if (TC_IN(o, nface, 1)) rw[o] = r;
        } else if (UPD == UPD_FE) {
          if (TC_IN(o, nface, 1)) ws[o] = R::fma(dt, r, cW0);
        } else {
          const T a = have_hist ? R::fma(T(1.5), r, R::mul(T(-0.5), hrw[kk])) : r;
          if (TC_IN(o, nface, 1)) ws[o] = R::fma(dt, a, cW0);
          if (TC_IN(o, nface, 1)) rw[o] = r;
        }
      }
    }
    // carry plane k+1 and the fluxes of face k+1
    pU0 = cU0; pV0 = cV0; pW0 = cW0;
    cU0 = nU0; cUxm = nUxm; cV0 = nV0; cVym = nVym;
    cW0 = nW0; cWxm = nWxm; cWxp = nWxp; cWym = nWym; cWyp = nWyp;
    Fuw_p = Fuw_p1; Fuw_m = Fuw_m1; Fvw_p = Fvw_p1; Fvw_m = Fvw_m1; Fww = Fww1;
  }
}

// FP64 storage: the stencils plane by plane, every flux formed where it is
// used (the registers that carrying values up the column would take cost
// the double-precision kernels more than the loads they save).  Same slot
// layout as rhs_march; no base profile (FP64 fields hold the total velocity).
template <bool FULL, int UPD, int KB, int HY, int HX>
__device__ __forceinline__ void rhs_planes(const Grid<double>& g, const double (*__restrict__ su)[HY][HX],
                                           const double (*__restrict__ sv)[HY][HX],
                                           const double (*__restrict__ sw)[HY][HX], int cx, int cy, int i, int j,
                                           bool active, int kb, double* __restrict__ us, double* __restrict__ vs,
                                           double* __restrict__ ws, double* __restrict__ ru, double* __restrict__ rv,
                                           double* __restrict__ rw, double (&hru)[KB], double (&hrv)[KB],
                                           double (&hrw)[KB], double forcing, double dt, int have_hist) {
  using T = double;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t plane = (size_t)nx * ny;
  const size_t ncell = plane * nz, nface = plane * (nz + 1);  // field extents (bounds-checked builds)
  (void)ncell; (void)nface;
  const T qx = T(0.25) * g.idx, qy = T(0.25) * g.idy;
#pragma unroll 1
  for (int kk = 0; kk < KB; ++kk) {
    const int k = kb + kk;
    if (k > nz) break;
    const int sm = kk, s0 = kk + 1, sp = kk + 2;
    if (active && k < nz) {
      const size_t o = (size_t)k * plane + (size_t)j * nx + i;
      const T idzf = g.idzf[k];
      const T qzf = T(0.25) * idzf;
      // ---------------- u at cell k ----------------
      {
        const T U0 = su[s0][cy][cx], Uxm = su[s0][cy][cx - 1], Uxp = su[s0][cy][cx + 1];
        const T Uym = su[s0][cy - 1][cx], Uyp = su[s0][cy + 1][cx];
        const T Uzm = su[sm][cy][cx], Uzp = su[sp][cy][cx];
        const bool edge = (i == nx - 1);
        T r = T(0);
        if (!(edge && g.rhs_fused)) {
          r = g.nu_idx2 * (Uxp - T(2) * U0 + Uxm) + g.nu_idy2 * (Uyp - T(2) * U0 + Uym);
          if (FULL) r += g.nu * ((Uzp - U0) * g.idzc[k + 1] - (U0 - Uzm) * g.idzc[k]) * idzf;
        }
        if (!edge) {
          const T duudx = (sq(U0 + Uxp) - sq(Uxm + U0)) * qx;
          const T vu_t = (sv[s0][cy][cx] + sv[s0][cy][cx + 1]) * (U0 + Uyp);
          const T vu_b = (sv[s0][cy - 1][cx] + sv[s0][cy - 1][cx + 1]) * (Uym + U0);
          const T wu_t = (sw[sp][cy][cx] + sw[sp][cy][cx + 1]) * (U0 + Uzp);
          const T wu_b = (sw[s0][cy][cx] + sw[s0][cy][cx + 1]) * (Uzm + U0);
          r -= duudx + (vu_t - vu_b) * qy + (wu_t - wu_b) * qzf;
        }
        if (UPD == UPD_RHS_ONLY) {
          if (TC_IN(o, ncell, 1)) ru[o] = r;
        } else if (UPD == UPD_FE) {
          T q = U0 + dt * r;
          if (TC_IN(o, ncell, 1)) us[o] = q + dt * T(1);
        } else {
          r += forcing;
          if (TC_IN(o, ncell, 1)) us[o] = have_hist ? U0 + dt * (T(1.5) * r - T(0.5) * hru[0]) : U0 + dt * r;
          if (TC_IN(o, ncell, 1)) ru[o] = r;
        }
      }
      // ---------------- v at cell k ----------------
      {
        const T V0 = sv[s0][cy][cx], Vxm = sv[s0][cy][cx - 1], Vxp = sv[s0][cy][cx + 1];
        const T Vym = sv[s0][cy - 1][cx], Vyp = sv[s0][cy + 1][cx];
        const T Vzm = sv[sm][cy][cx], Vzp = sv[sp][cy][cx];
        const bool edge = (j == ny - 1);
        T r = T(0);
        if (!(edge && g.rhs_fused)) {
          r = g.nu_idx2 * (Vxp - T(2) * V0 + Vxm) + g.nu_idy2 * (Vyp - T(2) * V0 + Vym);
          if (FULL) r += g.nu * ((Vzp - V0) * g.idzc[k + 1] - (V0 - Vzm) * g.idzc[k]) * idzf;
        }
        if (!edge) {
          const T uv_r = (su[s0][cy][cx] + su[s0][cy + 1][cx]) * (V0 + Vxp);
          const T uv_l = (su[s0][cy][cx - 1] + su[s0][cy + 1][cx - 1]) * (Vxm + V0);
          const T dvvdy = (sq(V0 + Vyp) - sq(Vym + V0)) * qy;
          const T wv_t = (sw[sp][cy][cx] + sw[sp][cy + 1][cx]) * (V0 + Vzp);
          const T wv_b = (sw[s0][cy][cx] + sw[s0][cy + 1][cx]) * (Vzm + V0);
          r -= (uv_r - uv_l) * qx + dvvdy + (wv_t - wv_b) * qzf;
        }
        if (UPD == UPD_RHS_ONLY) {
          if (TC_IN(o, ncell, 1)) rv[o] = r;
        } else if (UPD == UPD_FE) {
          if (TC_IN(o, ncell, 1)) vs[o] = V0 + dt * r;
        } else {
          if (TC_IN(o, ncell, 1)) vs[o] = have_hist ? V0 + dt * (T(1.5) * r - T(0.5) * hrv[0]) : V0 + dt * r;
          if (TC_IN(o, ncell, 1)) rv[o] = r;
        }
      }
    }
    // ---------------- w at face k ----------------
    if (active && k >= 1 && k <= nz - 1) {
      const size_t o = (size_t)k * plane + (size_t)j * nx + i;
      const T W0 = sw[s0][cy][cx], Wxm = sw[s0][cy][cx - 1], Wxp = sw[s0][cy][cx + 1];
      const T Wym = sw[s0][cy - 1][cx], Wyp = sw[s0][cy + 1][cx];
      const T Wzm = sw[sm][cy][cx], Wzp = sw[sp][cy][cx];
      T r = g.nu_idx2 * (Wxp - T(2) * W0 + Wxm) + g.nu_idy2 * (Wyp - T(2) * W0 + Wym);
      // z term of diffusion_w divides by dz_c[K-1] (operators.py:120,1025)
      if (FULL) r += g.nu * ((Wzp - W0) * g.idzf[k] - (W0 - Wzm) * g.idzf[k - 1]) * g.idzc[k - 1];
      const T uw_r = (su[sm][cy][cx] + su[s0][cy][cx]) * (W0 + Wxp);
      const T uw_l = (su[sm][cy][cx - 1] + su[s0][cy][cx - 1]) * (Wxm + W0);
      const T vw_t = (sv[sm][cy][cx] + sv[s0][cy][cx]) * (W0 + Wyp);
      const T vw_b = (sv[sm][cy - 1][cx] + sv[s0][cy - 1][cx]) * (Wym + W0);
      const T dwwdz = (sq(W0 + Wzp) - sq(Wzm + W0)) * (T(0.25) * g.idzc[k]);
      r -= (uw_r - uw_l) * qx + (vw_t - vw_b) * qy + dwwdz;
      if (UPD == UPD_RHS_ONLY) {
        if (TC_IN(o, nface, 1)) rw[o] = r;
      } else if (UPD == UPD_FE) {
        if (TC_IN(o, nface, 1)) ws[o] = W0 + dt * r;
      } else {
        if (TC_IN(o, nface, 1)) ws[o] = have_hist ? W0 + dt * (T(1.5) * r - T(0.5) * hrw[0]) : W0 + dt * r;
        if (TC_IN(o, nface, 1)) rw[o] = r;
      }
    }
#pragma unroll
    for (int q = 0; q + 1 < KB; ++q) {
      hru[q] = hru[q + 1]; hrv[q] = hrv[q + 1]; hrw[q] = hrw[q + 1];
    }
  }
}

// The stencils of a staged tile: rhs_march (FP32 storage) or rhs_planes (FP64).
template <class T, bool FULL, int UPD, int KB, int HY, int HX>
__device__ __forceinline__ void rhs_stencils(const Grid<T>& g, const T (*su)[HY][HX], const T (*sv)[HY][HX],
                                             const T (*sw)[HY][HX], int cx, int cy, int i, int j, bool active,
                                             int kb, T* us, T* vs, T* ws, T* ru, T* rv, T* rw, T (&hru)[KB],
                                             T (&hrv)[KB], T (&hrw)[KB], T forcing, T dt, int have_hist,
                                             const T* pre = nullptr) {
  if constexpr (sizeof(T) == 8)
    rhs_planes<FULL, UPD, KB, HY, HX>(g, su, sv, sw, cx, cy, i, j, active, kb, us, vs, ws, ru, rv, rw, hru, hrv, hrw,
                                      forcing, dt, have_hist);
  else
    rhs_march<T, FULL, UPD, KB, HY, HX>(g, su, sv, sw, cx, cy, i, j, active, kb, us, vs, ws, ru, rv, rw, hru, hrv,
                                        hrw, forcing, dt, have_hist, pre);
}

// The tile (bx, by, bz) of the block grid above; k_rhs_update runs one tile
// per block, the ensemble kernel of tc_batch.cuh loops over the tiles of all
// members (the shared tile is reused: callers separate tiles by a barrier).
template <class T, bool FULL, int UPD>
__device__ __forceinline__ void rhs_tile(const Grid<T>& g, const T* __restrict__ u, const T* __restrict__ v,
                                         const T* __restrict__ w, T* __restrict__ us, T* __restrict__ vs,
                                         T* __restrict__ ws, T* __restrict__ ru, T* __restrict__ rv,
                                         T* __restrict__ rw, const double* __restrict__ forcing_dev, T dt,
                                         int have_hist, int bx, int by, int bz) {
  constexpr int RHS_TY = rhs_ty<T>(), RHS_HY = RHS_TY + 2, RHS_NH = RHS_HX * RHS_HY;
  constexpr int RHS_KB = rhs_kb<T>();
  constexpr int RHS_NS = RHS_KB + 2;
  static_assert(RHS_NH <= 2 * RHS_TX * RHS_TY, "two halo elements per thread at most");
  __shared__ T su[RHS_NS][RHS_HY][RHS_HX];
  __shared__ T sv[RHS_NS][RHS_HY][RHS_HX];
  __shared__ T sw[RHS_NS][RHS_HY][RHS_HX];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t plane = (size_t)nx * ny;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * RHS_TX + tx;
  const int i0 = bx * RHS_TX, j0 = by * RHS_TY;
  const int i = i0 + tx, j = j0 + ty;
  const bool active = (i < nx) && (j < ny);
  const int kb = bz * RHS_KB;  // planes kb .. kb+RHS_KB-1 (<= nz)
  const T top = g.top_neumann ? T(1) : T(-1);
  const T forcing = (UPD == UPD_AB2) ? (T)(*forcing_dev) : T(0);
  // halo elements of this thread: e0 = tid, e1 = tid + block size (if < RHS_NH)
  const int e1 = tid + RHS_TX * RHS_TY;
  const bool has1 = e1 < RHS_NH;
  size_t off[2];
  int hyx[2][2];
  {
    const int es[2] = {tid, e1};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int hy = es[q] / RHS_HX, hx = es[q] - (es[q] / RHS_HX) * RHS_HX;
      int jj = j0 - 1 + hy, ii = i0 - 1 + hx;
      while (jj < 0) jj += ny;
      while (jj >= ny) jj -= ny;
      while (ii < 0) ii += nx;
      while (ii >= nx) ii -= nx;
      off[q] = (size_t)jj * nx + ii;
      hyx[q][0] = hy; hyx[q][1] = hx;
    }
  }
  // AB2 history of this thread's points, loaded with the staging so that
  // their latency overlaps it
  T pf_ru[RHS_KB], pf_rv[RHS_KB], pf_rw[RHS_KB];
#pragma unroll
  for (int q = 0; q < RHS_KB; ++q) {
    const int k = kb + q;
    const size_t o = (size_t)k * plane + (size_t)j * nx + i;
    const bool cell = active && k < nz, face = active && k >= 1 && k <= nz - 1;
    const bool hist = UPD == UPD_AB2 && have_hist;
    pf_ru[q] = (cell && hist) ? ru[o] : T(0);
    pf_rv[q] = (cell && hist) ? rv[o] : T(0);
    pf_rw[q] = (face && hist) ? rw[o] : T(0);
  }
  // stage planes p = kb-1 .. kb+RHS_KB into slots 0 .. RHS_NS-1 (stored
  // values; u / v z ghosts: sign * q[pc])
#pragma unroll
  for (int sl = 0; sl < RHS_NS; ++sl) {
    const int p = kb - 1 + sl;
    const int pc = p < 0 ? 0 : (p >= nz ? nz - 1 : p);
    const T sgn = p < 0 ? T(-1) : (p >= nz ? top : T(1));
    const bool wok = (p >= 0) && (p <= nz);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (q == 1 && !has1) break;
      const size_t oc = (size_t)pc * plane + off[q];
      const T uu = sgn * ldg(u + oc);
      const T vv = sgn * ldg(v + oc);
      const T ww = wok ? ldg(w + (size_t)p * plane + off[q]) : T(0);
      su[sl][hyx[q][0]][hyx[q][1]] = uu;
      sv[sl][hyx[q][0]][hyx[q][1]] = vv;
      sw[sl][hyx[q][0]][hyx[q][1]] = ww;
    }
  }
  __syncthreads();
  rhs_stencils<T, FULL, UPD, RHS_KB, RHS_HY, RHS_HX>(g, su, sv, sw, tx + 1, ty + 1, i, j, active, kb, us, vs, ws, ru,
                                                     rv, rw, pf_ru, pf_rv, pf_rw, forcing, dt, have_hist);
}

// FP32 storage: the compiler's own register choice (48 in the IMEX form, 5
// blocks per SM); bounding it to 5 blocks gives the same count and a slower
// schedule.
template <class T, bool FULL, int UPD>
__global__ void __launch_bounds__(RHS_TX * rhs_ty<T>()) k_rhs_update(Grid<T> g, const T* __restrict__ u,
                                                                const T* __restrict__ v, const T* __restrict__ w,
                                                                T* __restrict__ us, T* __restrict__ vs,
                                                                T* __restrict__ ws, T* __restrict__ ru,
                                                                T* __restrict__ rv, T* __restrict__ rw,
                                                                const double* __restrict__ forcing_dev, T dt,
                                                                int have_hist) {
  rhs_tile<T, FULL, UPD>(g, u, v, w, us, vs, ws, ru, rv, rw, forcing_dev, dt, have_hist, blockIdx.x, blockIdx.y,
                         blockIdx.z);
}

// FP64 storage: bounded to 4 blocks per SM (64 registers, no spills); left
// free the compiler takes 74 and 3 blocks fit.
template <bool FULL, int UPD>
__global__ void __launch_bounds__(RHS_TX * rhs_ty<double>(), 4) k_rhs_update_f64(
    Grid<double> g, const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
    double* __restrict__ us, double* __restrict__ vs, double* __restrict__ ws, double* __restrict__ ru,
    double* __restrict__ rv, double* __restrict__ rw, const double* __restrict__ forcing_dev, double dt,
    int have_hist) {
  rhs_tile<double, FULL, UPD>(g, u, v, w, us, vs, ws, ru, rv, rw, forcing_dev, dt, have_hist, blockIdx.x,
                              blockIdx.y, blockIdx.z);
}

// The RHS kernel for storage type T.
template <class T, bool FULL, int UPD> struct RhsKernel {
  static constexpr auto fn = k_rhs_update<T, FULL, UPD>;
};
template <bool FULL, int UPD> struct RhsKernel<double, FULL, UPD> {
  static constexpr auto fn = k_rhs_update_f64<FULL, UPD>;
};

// ---------------------------------------------------------------------------
// Crank-Nicolson tables.  Row m of a system:
//   a_m x_{m-1} + b_m x_m + c_m x_{m+1} = q_m + beta (cA_m s_{-1} + cB_m s_0 + cC_m s_{+1})
// u/v (operators.py:581-644): n = nz rows, row m <-> plane m, explicit
//   stencil on planes m-1, m, m+1 with the wall closures of :635-644.
// w (operators.py:753-803): n = nz-1 rows, row m <-> face m+1, explicit
//   stencil on faces m-1, m, m+1 (the reference's index convention).
// Thomas factors: inv_den_m = 1/(b_m - a_m cp_{m-1}), cp_m = c_m inv_den_m.
// Chunked sweep (rows split in chunks of L, 16 or 32): with f_m = -a_m inv_den_m,
// G_m = prod_{j = chunk start .. m} f_j and H_m = prod_{j = m .. chunk end}
// (-cp_j), a chunk swept from zero boundary values is corrected by
// d'_m += G_m d'_(start-1) and x_m += H_m x_(end+1).
// Table layout per system: 8 arrays of length nz: a, inv_den, cp, cA, cB, cC, G, H;
// after cn_fold, a holds f and cA, cB, cC the folded coefficients.
// ---------------------------------------------------------------------------
struct CnTab {
  double* uv;    // 8*nz
  double* w;     // 8*nz (first nz-1 rows used)
  double* beta;
  double* corr;  // nz: S(U0) - U0 of the u system (FP32-arithmetic sweeps of u - U0)
};

__device__ __forceinline__ void cn_chunk_products(double* a, double* iv, double* cp, double* G, double* H, int n,
                                                  int L) {
  for (int m = 0; m < n; ++m) {
    const double f = -a[m] * iv[m];
    G[m] = (m % L == 0) ? f : G[m - 1] * f;
  }
  for (int m = n - 1; m >= 0; --m) {
    const int e = min((m / L + 1) * L, n) - 1;
    H[m] = (m == e) ? -cp[m] : H[m + 1] * (-cp[m]);
  }
}

// Fold the explicit half and the forward elimination of a row into four
// coefficients, d'_m = eA s_{-1} + eB s_0 + eC s_{+1} + f d'_{m-1}, with
// f = -a_m rden_m, eX = rden_m (beta cX_m + [X is the row's own point]); the
// own point is s_0 for u/v and s_{+1} for w (stored over a, cA, cB, cC).
__device__ __forceinline__ void cn_fold_row(double* a, const double* iv, double* cA, double* cB, double* cC, int m,
                                            double beta, bool w_rows) {
  const double r = iv[m];
  a[m] = -a[m] * r;
  cA[m] = r * (beta * cA[m]);
  cB[m] = r * (beta * cB[m] + (w_rows ? 0.0 : 1.0));
  cC[m] = r * (beta * cC[m] + (w_rows ? 1.0 : 0.0));
}
__device__ __forceinline__ void cn_fold(double* a, const double* iv, double* cA, double* cB, double* cC, int n,
                                        double beta, bool w_rows) {
  for (int m = 0; m < n; ++m) cn_fold_row(a, iv, cA, cB, cC, m, beta, w_rows);
}

// CN image of the base profile minus itself (zero without a base), from the
// folded u / v rows: unchunked sweeps, FP64.
__device__ __forceinline__ void cn_base_corr(const CnTab& t, int nz, const double* __restrict__ ubase) {
  const double* a = t.uv; const double* cp = a + 2 * nz;
  const double* cA = a + 3 * nz; const double* cB = cA + nz; const double* cC = cB + nz;
  if (ubase) {
    double dp = 0.0;
    for (int m = 0; m < nz; ++m) {
      const double sm = m > 0 ? ubase[m - 1] : 0.0, sp = m + 1 < nz ? ubase[m + 1] : 0.0;
      dp = a[m] * dp + (cA[m] * sm + cB[m] * ubase[m] + cC[m] * sp);
      t.corr[m] = dp;
    }
    double x = 0.0;
    for (int m = nz - 1; m >= 0; --m) {
      x = t.corr[m] - cp[m] * x;
      t.corr[m] = x - ubase[m];
    }
  } else {
    for (int m = 0; m < nz; ++m) t.corr[m] = 0.0;
  }
}

// Rows of the CN systems at level m (operators.py:581-644 for u / v,
// 753-803 for w): the implicit row (am, bm, cm) with the wall closures and
// the explicit half's stencil (ea, eb, ec).
struct CnRow { double am, bm, cm, ea, eb, ec; };
__device__ __forceinline__ CnRow cn_row_uv(const double* __restrict__ dzf, const double* __restrict__ dzc, int m,
                                           int nz, double alpha, int top_neumann) {
  CnRow r;
  double dl = dzc[m], dr = dzc[m + 1], dc = dzf[m];
  double lo = -alpha / (dl * dc);
  double ce = 1.0 + alpha * (1.0 / dl + 1.0 / dr) / dc;
  double up = -alpha / (dr * dc);
  r.am = lo; r.bm = ce; r.cm = up;
  if (m == 0) { r.am = 0.0; r.bm = ce - lo; }
  if (m == nz - 1) { r.bm = top_neumann ? ce + up : ce - up; r.cm = 0.0; }
  // explicit half (operators.py:635-644)
  r.ea = 1.0 / (dl * dc); r.eb = -(1.0 / dr + 1.0 / dl) / dc; r.ec = 1.0 / (dr * dc);
  if (m == 0) { r.ea = 0.0; r.eb = (-1.0 / dr - 2.0 / dl) / dc; }
  if (m == nz - 1) {
    if (top_neumann) { r.eb = -1.0 / (dl * dc); }
    else { r.eb = (-2.0 / dr - 1.0 / dl) / dc; }
    r.ec = 0.0;
  }
  return r;
}
__device__ __forceinline__ CnRow cn_row_w(const double* __restrict__ dzf, const double* __restrict__ dzc, int m,
                                          int n, double alpha) {
  CnRow r;
  double dl = dzf[m], dr = dzf[m + 1], dcv = dzc[m + 1];
  double lo = -alpha / (dl * dcv);
  double ce = 1.0 + alpha * (1.0 / dl + 1.0 / dr) / dcv;
  double up = -alpha / (dr * dcv);
  r.am = (m == 0) ? 0.0 : lo; r.bm = ce; r.cm = (m == n - 1) ? 0.0 : up;
  r.ea = 1.0 / (dl * dcv); r.eb = -(1.0 / dr + 1.0 / dl) / dcv; r.ec = 1.0 / (dr * dcv);
  if (m == 0) r.ea = 0.0;
  if (m == n - 1) r.ec = 0.0;
  return r;
}

// The CN tables of the u / v system (t.uv, and t.corr: the CN image of the
// base profile minus itself) and of the w system (t.w), for time step dt and
// chunk length L.  staged != 0: the block works in dynamic shared memory
// (8 nz + 8 nz + nz doubles): every thread forms rows of both systems, one
// thread per system runs the Thomas factor recurrence (its only sequential
// part), the chunk products, the fold and the base profile's sweeps follow,
// and the block copies the tables out.  staged == 0: one thread per system
// does everything in the tables themselves.  The same operations on the same
// values either way.
__global__ void k_cn_tables(CnTab t, const double* __restrict__ dzf, const double* __restrict__ dzc, int nz,
                            double nu, double dt, int top_neumann, int L, const double* __restrict__ ubase,
                            int staged) {
  const double theta = 0.5;
  const double alpha = theta * dt * nu;
  const double beta = (1.0 - theta) * dt * nu;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = nz - 1;  // rows of the w system
  extern __shared__ double cn_sm[];
  CnTab g = t;  // where the builds write
  if (staged) {
    g.uv = cn_sm;
    g.w = cn_sm + 8 * nz;
    g.corr = cn_sm + 16 * nz;
    for (int e = tid; e < 17 * nz; e += nthr) cn_sm[e] = 0.0;
    __syncthreads();
    // rows: a <- am, iv <- bm, cp <- cm until the recurrence replaces them
    for (int m = tid; m < nz; m += nthr) {
      const CnRow r = cn_row_uv(dzf, dzc, m, nz, alpha, top_neumann);
      double* u = g.uv;
      u[m] = r.am; u[nz + m] = r.bm; u[2 * nz + m] = r.cm;
      u[3 * nz + m] = r.ea; u[4 * nz + m] = r.eb; u[5 * nz + m] = r.ec;
      if (m < n) {
        const CnRow q = cn_row_w(dzf, dzc, m, n, alpha);
        double* w = g.w;
        w[m] = q.am; w[nz + m] = q.bm; w[2 * nz + m] = q.cm;
        w[3 * nz + m] = q.ea; w[4 * nz + m] = q.eb; w[5 * nz + m] = q.ec;
      }
    }
    __syncthreads();
    if (tid < 2) {
      double* a = tid == 0 ? g.uv : g.w;
      double* iv = a + nz; double* cp = iv + nz;
      const int rows = tid == 0 ? nz : n;
      double cprev = 0.0;
      for (int m = 0; m < rows; ++m) {
        const double den = iv[m] - a[m] * cprev;
        const double rden = 1.0 / den;
        iv[m] = rden; cp[m] = cp[m] * rden; cprev = cp[m];
      }
    }
    __syncthreads();
    if (tid < 2) {
      double* a = tid == 0 ? g.uv : g.w;
      double* iv = a + nz; double* cp = iv + nz;
      double* cC = cp + 3 * nz;
      cn_chunk_products(a, iv, cp, cC + nz, cC + 2 * nz, tid == 0 ? nz : n, L);
    }
    __syncthreads();
    for (int m = tid; m < nz; m += nthr) {
      double* a = g.uv; double* iv = a + nz; double* cA = a + 3 * nz;
      cn_fold_row(a, iv, cA, cA + nz, cA + 2 * nz, m, beta, false);
      if (m < n) {
        double* aw = g.w; double* ivw = aw + nz; double* cAw = aw + 3 * nz;
        cn_fold_row(aw, ivw, cAw, cAw + nz, cAw + 2 * nz, m, beta, true);
      }
    }
    __syncthreads();
    if (tid == 0) {
      *t.beta = beta;
      cn_base_corr(g, nz, ubase);
    }
    __syncthreads();
    for (int e = tid; e < 8 * nz; e += nthr) {
      t.uv[e] = cn_sm[e];
      t.w[e] = cn_sm[8 * nz + e];
    }
    for (int e = tid; e < nz; e += nthr) t.corr[e] = cn_sm[16 * nz + e];
    return;
  }
  if (tid == 0) {
    double* a = t.uv; double* iv = a + nz; double* cp = iv + nz;
    double* cA = cp + nz; double* cB = cA + nz; double* cC = cB + nz;
    double cprev = 0.0;
    for (int m = 0; m < nz; ++m) {
      const CnRow r = cn_row_uv(dzf, dzc, m, nz, alpha, top_neumann);
      const double den = r.bm - r.am * cprev;
      const double rden = 1.0 / den;
      a[m] = r.am; iv[m] = rden; cp[m] = r.cm * rden; cprev = cp[m];
      cA[m] = r.ea; cB[m] = r.eb; cC[m] = r.ec;
    }
    cn_chunk_products(a, iv, cp, cC + nz, cC + 2 * nz, nz, L);
    *t.beta = beta;
    cn_fold(a, iv, cA, cB, cC, nz, beta, false);
    cn_base_corr(t, nz, ubase);
  } else if (tid == 1) {
    double* a = t.w; double* iv = a + nz; double* cp = iv + nz;
    double* cA = cp + nz; double* cB = cA + nz; double* cC = cB + nz;
    double cprev = 0.0;
    for (int m = 0; m < n; ++m) {
      const CnRow r = cn_row_w(dzf, dzc, m, n, alpha);
      const double den = r.bm - r.am * cprev;
      const double rden = 1.0 / den;
      a[m] = r.am; iv[m] = rden; cp[m] = r.cm * rden; cprev = cp[m];
      cA[m] = r.ea; cB[m] = r.eb; cC[m] = r.ec;
    }
    cn_chunk_products(a, iv, cp, cC + nz, cC + 2 * nz, n, L);
    cn_fold(a, iv, cA, cB, cC, n, beta, true);
  }
}

// ---------------------------------------------------------------------------
// Kernel (b): batched tridiagonal solve of the CN systems
// (solve_implicit_diffusion_u/v/w, operators.py:563-811; the reference's PCR,
// tridiag.py:33-58, solves the same systems).  A block owns 32*VEC
// consecutive columns of one component (blockIdx.z = 0 u, 1 v, 2 w) and one
// warp per chunk of L rows; a thread owns VEC adjacent columns (VEC = 2 for
// FP32 storage: 8-byte loads).  Each thread loads the L + 2 planes its
// chunk's stencil needs straight into registers (coalesced across the warp,
// all loads in flight together), sweeps the chunk forward and backward from
// zero boundary values, and the chunk ends are stitched with one value per
// chunk boundary (G/H tables).  Every value is read and written once; the
// arithmetic is FP64 (u with its base profile added).
// ---------------------------------------------------------------------------
template <class T, int VEC> struct CnVec;
template <> struct CnVec<double, 1> {
  static __device__ __forceinline__ void ld(const double* p, double (&o)[1]) { o[0] = *p; }
  template <class A> static __device__ __forceinline__ void st(double* p, const A (&o)[1]) { *p = (double)o[0]; }
};
template <> struct CnVec<float, 1> {
  static __device__ __forceinline__ void ld(const float* p, float (&o)[1]) { o[0] = *p; }
  template <class A> static __device__ __forceinline__ void st(float* p, const A (&o)[1]) { *p = (float)o[0]; }
};
template <> struct CnVec<float, 2> {
  static __device__ __forceinline__ void ld(const float* p, float (&o)[2]) {
    const float2 x = *reinterpret_cast<const float2*>(p);
    o[0] = x.x; o[1] = x.y;
  }
  template <class A> static __device__ __forceinline__ void st(float* p, const A (&o)[2]) {
    *reinterpret_cast<float2*>(p) = make_float2((float)o[0], (float)o[1]);
  }
};
// Arithmetic of the sweeps: FP64 for FP64 storage; FP32 for FP32 storage,
// where u is solved as its stored deviation u - U0 (the system is linear:
// S(u' + U0) - U0 = S(u') + (S(U0) - U0), the last column tabulated in FP64
// by k_cn_tables as CnTab::corr) so that no FP32 sum carries the O(1) base.
template <class T> struct CnArith { using type = double; };
template <> struct CnArith<float> { using type = float; };

// Column block bx of component comp (the block grid above), chunks of Lr <= L
// rows (the tables' chunk length; L sizes the register windows; FIXED: Lr is
// L, known at compile time); blockDim.y may exceed the chunks of this
// system, the extra warps only take part in the barriers.
template <class T, int L, int VEC, bool FIXED = false>
__device__ __forceinline__ void cn_tile(T* __restrict__ u, T* __restrict__ v, T* __restrict__ w, const CnTab& t,
                                        const double* __restrict__ ubase, int nx, int ny, int nz, int bx, int comp,
                                        int Lr_arg) {
  using A = typename CnArith<T>::type;
  constexpr bool F32 = sizeof(A) == 4;
  // FP32 sweeps of two columns per thread: packed FP32x2 arithmetic
  constexpr bool PK = F32 && VEC == 2;
  const int Lr = FIXED ? L : Lr_arg;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x, chunk = threadIdx.y, nchunk = blockDim.y;
  const int tid = chunk * 32 + lane, nthr = 32 * nchunk;
  A* tab = reinterpret_cast<A*>(smraw);                      // 8*nz
  A* shb = tab + 8 * nz;                                     // nz: base (FP64) or its CN correction (FP32), u only
  A* bnd = shb + nz;                                         // 2 * nchunk * 32 * VEC
  const double* src = comp == 2 ? t.w : t.uv;
  for (int e = tid; e < 8 * nz; e += nthr) tab[e] = (A)src[e];
  for (int e = tid; e < nz; e += nthr)
    shb[e] = (comp == 0 && ubase) ? (A)(F32 ? t.corr[e] : ubase[e]) : A(0);
  // nx*ny is even, so with VEC = 2 a pair of columns is valid as a whole
  const int col = (bx * 32 + lane) * VEC;
  const int ncols = nx * ny;
  const bool colok = col < ncols;
  T* q = (comp == 0 ? u : (comp == 1 ? v : w)) + (colok ? col : 0);
  // extent of the field from q (bounds-checked builds)
  const size_t qn = (size_t)ncols * (comp < 2 ? nz : nz + 1) - (colok ? col : 0);
  (void)qn;
  const int n = comp < 2 ? nz : nz - 1;
  const int s0 = chunk * Lr, e0 = min(s0 + Lr, n);          // rows [s0, e0)
  const bool act = s0 < n;
  // window: stencil sources of rows s0..e0-1 = planes (u/v) or faces (w)
  // s0-1 .. e0; row m uses wv[m-s0], wv[m-s0+1], wv[m-s0+2]; the unknown of
  // row m is plane m (u/v: wv[m-s0+1]) or face m+1 (w: wv[m-s0+2])
  T wv[L + 2][VEC];
  const int plmax = comp < 2 ? nz - 1 : nz;
  // FP64 storage ("lean" addressing, measured 57 -> 53 us at 192x192x128):
  // window entries [wlo, whi) exist (entry tt is plane s0-1+tt), rows
  // s0 .. s0+nrow-1 are this chunk's, offsets within a field in 32 bits (a
  // field has fewer than 2^32 elements) stepped by one plane per entry, and
  // every entry is loaded (an absent one from the column's first plane) and
  // then kept or zeroed, so that the loads issue back to back.  FP32 storage
  // keeps the 64-bit plane products and per-entry guards, which measured
  // faster there (32 vs 35 us).
  constexpr bool LEAN = sizeof(T) == 8;
  const int wlo = s0 >= 1 ? 0 : 1;
  const int whi = (act && colok) ? min(Lr + 2, plmax - s0 + 2) : 0;
  const int nrow = e0 - s0;
  const unsigned ucols = (unsigned)ncols;
  const size_t plane = (size_t)ncols;
  if constexpr (LEAN) {
    unsigned ow = (unsigned)(s0 - 1) * ucols;  // wraps for s0 = 0, whose entry 0 is not read
#pragma unroll
    for (int tt = 0; tt < L + 2; ++tt) {
      const bool ok = tt >= wlo && tt < whi;
      T x[VEC];
      if (TC_IN(ok ? ow : 0u, qn, VEC)) CnVec<T, VEC>::ld(q + (ok ? ow : 0u), x);
      else {
#pragma unroll
        for (int c = 0; c < VEC; ++c) x[c] = T(0);
      }
#pragma unroll
      for (int c = 0; c < VEC; ++c) wv[tt][c] = ok ? x[c] : T(0);
      ow += ucols;
    }
  } else {
#pragma unroll
    for (int tt = 0; tt < L + 2; ++tt) {
      const int pl = s0 - 1 + tt;
      if (act && colok && pl >= 0 && pl <= plmax && tt < Lr + 2 && TC_IN((size_t)pl * plane, qn, VEC)) {
        CnVec<T, VEC>::ld(q + (size_t)pl * plane, wv[tt]);
      } else {
#pragma unroll
        for (int c = 0; c < VEC; ++c) wv[tt][c] = T(0);
      }
    }
  }
  __syncthreads();  // tables staged
  const A* a = tab; const A* iv = a + nz; const A* cp = iv + nz;
  const A* cA = cp + nz; const A* cB = cA + nz; const A* cC = cB + nz;
  const A* G = cC + nz; const A* H = G + nz;
  (void)iv;
  // base profile of window entry tt (FP64 sweeps of u: planes in range; else 0)
  auto wb = [&](int tt) -> A {
    if constexpr (F32) {
      return A(0);
    } else {
      const int pl = s0 - 1 + tt;
      return (comp < 2 && pl >= 0 && pl < nz) ? shb[pl] : A(0);
    }
  };
  A y[L][VEC];
  A yend[VEC];
#pragma unroll
  for (int c = 0; c < VEC; ++c) yend[c] = A(0);
  if (act) {
    A yp[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) yp[c] = A(0);
    A bm = wb(0), bc = wb(1);
#pragma unroll
    for (int tt = 0; tt < L; ++tt) {
      const int m = s0 + tt;
      if (LEAN ? tt < nrow : m < e0) {
        const A bp = wb(tt + 2);
        const A f = a[m], ea = cA[m], eb = cB[m], ec = cC[m];
        if constexpr (PK) {
          // both columns in one packed FP32 operation (the same roundings);
          // FP32 sweeps carry no base (bm = bc = bp = 0)
          const float2 E = __ffma2_rn(make_float2(ea, ea), make_float2(wv[tt][0], wv[tt][1]),
                                      __ffma2_rn(make_float2(eb, eb), make_float2(wv[tt + 1][0], wv[tt + 1][1]),
                                                 __fmul2_rn(make_float2(ec, ec),
                                                            make_float2(wv[tt + 2][0], wv[tt + 2][1]))));
          const float2 Y = __ffma2_rn(make_float2(f, f), make_float2(yp[0], yp[1]), E);
          yp[0] = Y.x; yp[1] = Y.y;
          y[tt][0] = Y.x; y[tt][1] = Y.y;
        } else {
#pragma unroll
          for (int c = 0; c < VEC; ++c) {
            const A sm = (A)wv[tt][c] + bm, sc = (A)wv[tt + 1][c] + bc, sp = (A)wv[tt + 2][c] + bp;
            // the explicit part first: one dependent FMA per row on the recurrence
            const A E = fma(ea, sm, fma(eb, sc, ec * sp));
            yp[c] = fma(f, yp[c], E);
            y[tt][c] = yp[c];
          }
        }
        bm = bc; bc = bp;
      }
    }
#pragma unroll
    for (int c = 0; c < VEC; ++c) yend[c] = yp[c];
  }
#pragma unroll
  for (int c = 0; c < VEC; ++c) bnd[(chunk * VEC + c) * 32 + lane] = yend[c];
  __syncthreads();
  // true d' entering this chunk: scan the chunk ends below it
  A Din[VEC];
#pragma unroll
  for (int c = 0; c < VEC; ++c) Din[c] = A(0);
  for (int k = 0; k < chunk; ++k) {
    const A g = G[min(k * Lr + Lr, n) - 1];
#pragma unroll
    for (int c = 0; c < VEC; ++c) Din[c] = bnd[(k * VEC + c) * 32 + lane] + g * Din[c];
  }
  A zstart[VEC];
#pragma unroll
  for (int c = 0; c < VEC; ++c) zstart[c] = A(0);
  if (act) {
    // backward from a zero value beyond the chunk end, with the d' shift
    A zn[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) zn[c] = A(0);
#pragma unroll
    for (int tt = L - 1; tt >= 0; --tt) {
      const int m = s0 + tt;
      if (LEAN ? tt < nrow : m < e0) {
        const A g = G[m], cpm = cp[m];
        if constexpr (PK) {
          const float2 t = __ffma2_rn(make_float2(g, g), make_float2(Din[0], Din[1]), make_float2(y[tt][0], y[tt][1]));
          const float2 z = __ffma2_rn(make_float2(-cpm, -cpm), make_float2(zn[0], zn[1]), t);
          zn[0] = z.x; zn[1] = z.y;
          y[tt][0] = z.x; y[tt][1] = z.y;
        } else {
#pragma unroll
          for (int c = 0; c < VEC; ++c) {
            zn[c] = (y[tt][c] + g * Din[c]) - cpm * zn[c];
            y[tt][c] = zn[c];
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < VEC; ++c) zstart[c] = zn[c];
  }
#pragma unroll
  for (int c = 0; c < VEC; ++c) bnd[((nchunk + chunk) * VEC + c) * 32 + lane] = zstart[c];
  __syncthreads();
  // true x just beyond this chunk: scan the chunk starts above it
  A Xin[VEC];
#pragma unroll
  for (int c = 0; c < VEC; ++c) Xin[c] = A(0);
  for (int k = nchunk - 1; k > chunk; --k) {
    const int cs = k * Lr;
    if (cs < n) {
      const A h = H[cs];
#pragma unroll
      for (int c = 0; c < VEC; ++c) Xin[c] = bnd[((nchunk + k) * VEC + c) * 32 + lane] + h * Xin[c];
    }
  }
  if (act && colok) {
    unsigned os = (unsigned)(comp < 2 ? s0 : s0 + 1) * ucols;  // plane (u/v) or face (w) of row s0
#pragma unroll
    for (int tt = 0; tt < L; ++tt) {
      const int m = s0 + tt;
      if (LEAN ? tt < nrow : m < e0) {
        const A h = H[m];
        const A bs = comp < 2 ? shb[m] : A(0);
        A o[VEC];
        if constexpr (PK) {
          const float2 r = __fadd2_rn(
              __ffma2_rn(make_float2(h, h), make_float2(Xin[0], Xin[1]), make_float2(y[tt][0], y[tt][1])),
              make_float2(bs, bs));
          o[0] = r.x; o[1] = r.y;
        } else {
#pragma unroll
          for (int c = 0; c < VEC; ++c) o[c] = F32 ? (y[tt][c] + h * Xin[c]) + bs : (y[tt][c] + h * Xin[c]) - bs;
        }
        const int pl = comp < 2 ? m : m + 1;
        if (TC_IN(LEAN ? (size_t)os : (size_t)pl * plane, qn, VEC))
          CnVec<T, VEC>::st(LEAN ? q + os : q + (size_t)pl * plane, o);
      }
      os += ucols;
    }
  }
}

template <class T, int L, int VEC, int MAXT, bool FIXED>
__global__ void __launch_bounds__(MAXT) k_cn_solve(T* __restrict__ u, T* __restrict__ v, T* __restrict__ w,
                                                   CnTab t, const double* __restrict__ ubase, int nx, int ny,
                                                   int nz, int Lr) {
  cn_tile<T, L, VEC, FIXED>(u, v, w, t, ubase, nx, ny, nz, blockIdx.x, blockIdx.z, Lr);
}

// FP32 storage, two columns a thread (the packed sweeps): registers bounded
// to 64, four 256-thread blocks per SM (left free the sweeps take 95
// registers and half the resident blocks).
template <int L, int MAXT, bool FIXED>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT) k_cn_solve_pk(float* __restrict__ u, float* __restrict__ v,
                                                                 float* __restrict__ w, CnTab t,
                                                                 const double* __restrict__ ubase, int nx, int ny,
                                                                 int nz, int Lr) {
  cn_tile<float, L, 2, FIXED>(u, v, w, t, ubase, nx, ny, nz, blockIdx.x, blockIdx.z, Lr);
}

// Scalars slot layout (FP64, device).
enum : int {
  SC_FORCING = 0,
  SC_UBULK = 1,
  SC_DTI = 2,
  SC_MAXDIV = 3,
  SC_UTAU_BOT = 4,
  SC_UTAU_TOP = 5,
  SC_NONFINITE = 6,
  SC_COUNT = 8
};

// Deterministic final reduction of `n` bulk partials and the PI forcing update
// forcing += (U_b - u_b)/dt * 0.1 (solver.py:701-708), done by one block.
__device__ __forceinline__ void bulk_reduce_block(const double* partials, int n, double* scal, double scale,
                                                  double U_target, double dt, int update_forcing, double* sh) {
  const int t = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
  double a8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int e = t;
  for (; e + 7 * nt < n; e += 8 * nt) {
#pragma unroll
    for (int q = 0; q < 8; ++q) a8[q] += __ldcg(partials + e + q * nt);
  }
  for (; e < n; e += nt) a8[0] += __ldcg(partials + e);
  double acc = ((a8[0] + a8[1]) + (a8[2] + a8[3])) + ((a8[4] + a8[5]) + (a8[6] + a8[7]));
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double ub = s * scale;
    scal[SC_UBULK] = ub;
    if (update_forcing) scal[SC_FORCING] += (U_target - ub) / dt * 0.1;
  }
}

struct BulkArgs {
  double* partials;
  unsigned int* ticket;  // zero between launches; the last block resets it
  double* scal;
  double scale, U_target, dt;
  int update_forcing;
};

// ---------------------------------------------------------------------------
// Kernel (d): projection u -= dt grad p (projection.py:143-165), in place,
// fused with the bulk velocity (utils.py:207-223: sum of u dz_f dx dy / V over
// all DOFs) and the PI forcing update.  Each thread owns two x-adjacent points
// of one plane and moves them with 2-wide vector loads/stores; every block
// writes one partial sum and the last block to finish reduces them in a fixed
// order.  p is FP64.  nx is even, so the pairs never straddle a row.
// ---------------------------------------------------------------------------
#define PROJ_PK 16  // planes per block of k_project_bulk
template <class T> struct Vec2;
template <> struct Vec2<double> { using t = double2; };
template <> struct Vec2<float> { using t = float2; };

// Sources of the pressure the projection applies.  PSrc64: an FP64 p (out,
// when set, receives p rounded to FP32 as the base of a following
// single-precision Poisson step).
// pair(o) = p at o and o + 1, one(o) = p at o, keep(o, P) stores the pair P
// the thread applied at its own points.
struct PSrc64 {
  const double* p;
  float* out;
  __device__ __forceinline__ double2 pair(size_t o) const { return *reinterpret_cast<const double2*>(p + o); }
  __device__ __forceinline__ double one(size_t o) const { return ldg(p + o); }
  __device__ __forceinline__ void keep(size_t o, double2 P) const {
    if (out) *reinterpret_cast<float2*>(out + o) = make_float2((float)P.x, (float)P.y);
  }
};

// PSrcInc: the single-precision Poisson step's base p_b plus its increment
// dp, both FP32 and summed in FP64 (the gradient of p_b + dp is exact to FP64
// rounding, whatever the FP32 rounding of p_b); out receives p_b + dp
// rounded to FP32, the next step's base.
struct PSrcInc {
  const float* pb;
  const float* dp;
  float* out;
  __device__ __forceinline__ double2 pair(size_t o) const {
    const float2 a = *reinterpret_cast<const float2*>(pb + o), b = *reinterpret_cast<const float2*>(dp + o);
    return make_double2((double)a.x + (double)b.x, (double)a.y + (double)b.y);
  }
  __device__ __forceinline__ double one(size_t o) const { return (double)ldg(pb + o) + (double)ldg(dp + o); }
  __device__ __forceinline__ void keep(size_t o, double2 P) const {
    *reinterpret_cast<float2*>(out + o) = make_float2((float)P.x, (float)P.y);
  }
};

// Block (bx, by, bz) of a grid of gx x gy x gz blocks of 32 x 8 threads.
template <class T, class PS>
__device__ __forceinline__ void project_tile_ps(const Grid<T>& g, T* __restrict__ u, T* __restrict__ v,
                                                T* __restrict__ w, const PS& ps, double dt,
                                                const double* __restrict__ dzf, const BulkArgs& ba, int bx, int by,
                                                int bz, int gx, int gy, int gz) {
  using V2 = typename Vec2<T>::t;
  __shared__ double sh[32];
  __shared__ int last;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = 2 * (bx * 32 + threadIdx.x);
  const int j = by * 8 + threadIdx.y;
  const int k0 = bz * PROJ_PK;  // planes k0 .. k0+PROJ_PK-1
  const size_t ncell = (size_t)nx * ny * nz, nface = (size_t)nx * ny * (nz + 1);  // extents (bounds-checked builds)
  (void)ncell; (void)nface;
  // the accesses of plane k (pairs at o and at the y neighbour, the x neighbour of the pair)
  auto plane_in = [&](int k, int jp, int ipp) {
    return TC_IN(pidx(k, j, i, ny, nx), ncell, 2) && TC_IN(pidx(k, jp, i, ny, nx), ncell, 2) &&
           TC_IN(pidx(k, j, ipp, ny, nx), ncell, 1);
  };
  double acc = 0.0;
  if (i < nx && j < ny) {
    const int jp = wrap(j + 1, ny), ipp = wrap(i + 2, nx);
    const double cx = dt * (double)g.idx, cy = dt * (double)g.idy;
    // p of the plane below k0 for w's face k0 (walls excluded below)
    double2 Pm = make_double2(0.0, 0.0);
    if (k0 >= 1) Pm = ps.pair(pidx(k0 - 1, j, i, ny, nx));
    if constexpr (sizeof(T) == 4) {
      // FP32 storage: the next plane's loads are issued before this plane's
      // stores (the FP64 form has no registers to spare for it)
      struct Ld { double2 P, Py; double P2; V2 uu, vv, ww; };
      auto load = [&](int k) {
        Ld l;
        const size_t o = pidx(k, j, i, ny, nx);
        if (!plane_in(k, jp, ipp)) {
          l = Ld{};
          return l;
        }
        l.P = ps.pair(o);
        l.P2 = ps.one(pidx(k, j, ipp, ny, nx));
        l.Py = ps.pair(pidx(k, jp, i, ny, nx));
        l.uu = *reinterpret_cast<const V2*>(u + o);
        l.vv = *reinterpret_cast<const V2*>(v + o);
        l.ww = *reinterpret_cast<const V2*>(w + o);
        return l;
      };
      Ld cur = load(min(k0, nz - 1));
#pragma unroll
      for (int kk = 0; kk < PROJ_PK; ++kk) {
        const int k = k0 + kk;
        if (k < nz) {
          Ld nxt = cur;
          if (kk + 1 < PROJ_PK && k + 1 < nz) nxt = load(k + 1);
          const size_t o = pidx(k, j, i, ny, nx);
          const double2 P = cur.P, Py = cur.Py;
          const double P2 = cur.P2;
          V2 uu = cur.uu, vv = cur.vv;
          uu.x = (T)((double)uu.x - cx * (P.y - P.x));
          uu.y = (T)((double)uu.y - cx * (P2 - P.y));
          vv.x = (T)((double)vv.x - cy * (Py.x - P.x));
          vv.y = (T)((double)vv.y - cy * (Py.y - P.y));
          if (TC_IN(o, ncell, 2)) {
            *reinterpret_cast<V2*>(u + o) = uu;
            *reinterpret_cast<V2*>(v + o) = vv;
          }
          acc += ((double)uu.x + (double)uu.y + (g.ubase_d ? 2.0 * g.ubase_d[k] : 0.0)) * dzf[k];
          if (k >= 1) {
            const double cz = dt * (double)g.idzc[k];
            V2 ww = cur.ww;
            ww.x = (T)((double)ww.x - cz * (P.x - Pm.x));
            ww.y = (T)((double)ww.y - cz * (P.y - Pm.y));
            if (TC_IN(o, nface, 2)) *reinterpret_cast<V2*>(w + o) = ww;
          }
          ps.keep(o, P);
          Pm = P;
          cur = nxt;
        }
      }
    } else {
#pragma unroll
      for (int kk = 0; kk < PROJ_PK; ++kk) {
        const int k = k0 + kk;
        if (k < nz && plane_in(k, jp, ipp)) {
          const size_t o = pidx(k, j, i, ny, nx);
          const double2 P = ps.pair(o);
          const double P2 = ps.one(pidx(k, j, ipp, ny, nx));
          const double2 Py = ps.pair(pidx(k, jp, i, ny, nx));
          V2 uu = *reinterpret_cast<V2*>(u + o);
          V2 vv = *reinterpret_cast<V2*>(v + o);
          uu.x = (T)((double)uu.x - cx * (P.y - P.x));
          uu.y = (T)((double)uu.y - cx * (P2 - P.y));
          vv.x = (T)((double)vv.x - cy * (Py.x - P.x));
          vv.y = (T)((double)vv.y - cy * (Py.y - P.y));
          *reinterpret_cast<V2*>(u + o) = uu;
          *reinterpret_cast<V2*>(v + o) = vv;
          acc += ((double)uu.x + (double)uu.y + (g.ubase_d ? 2.0 * g.ubase_d[k] : 0.0)) * dzf[k];
          if (k >= 1) {
            const double cz = dt * (double)g.idzc[k];
            V2 ww = *reinterpret_cast<V2*>(w + o);
            ww.x = (T)((double)ww.x - cz * (P.x - Pm.x));
            ww.y = (T)((double)ww.y - cz * (P.y - Pm.y));
            *reinterpret_cast<V2*>(w + o) = ww;
          }
          ps.keep(o, P);
          Pm = P;
        }
      }
    }
  }
  double s = block_sum(acc, sh);
  const int nb = gx * gy * gz;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    ba.partials[((size_t)bz * gy + by) * gx + bx] = s;
    __threadfence();
    unsigned int t = atomicAdd(ba.ticket, 1u);
    last = (t == (unsigned)nb - 1u);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    bulk_reduce_block(ba.partials, nb, ba.scal, ba.scale, ba.U_target, ba.dt, ba.update_forcing, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) *ba.ticket = 0u;
  }
}

// The projection with an FP64 pressure p.
template <class T>
__device__ __forceinline__ void project_tile(const Grid<T>& g, T* __restrict__ u, T* __restrict__ v,
                                             T* __restrict__ w, const double* __restrict__ p, double dt,
                                             const double* __restrict__ dzf, const BulkArgs& ba, int bx, int by,
                                             int bz, int gx, int gy, int gz) {
  project_tile_ps<T, PSrc64>(g, u, v, w, PSrc64{p, nullptr}, dt, dzf, ba, bx, by, bz, gx, gy, gz);
}

template <class T, class PS>
__global__ void __launch_bounds__(256) k_project_bulk(Grid<T> g, T* __restrict__ u, T* __restrict__ v,
                                                      T* __restrict__ w, PS ps, double dt,
                                                      const double* __restrict__ dzf, BulkArgs ba) {
  project_tile_ps<T, PS>(g, u, v, w, ps, dt, dzf, ba, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y,
                         gridDim.z);
}

// Bulk sum over all DOFs without projection (set-up and diagnostics).
template <class T>
__global__ void __launch_bounds__(256) k_bulk_partials(Grid<T> g, const T* __restrict__ u,
                                                       const double* __restrict__ dzf,
                                                       double* __restrict__ partials) {
  __shared__ double sh[32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  double acc = 0.0;
  if (i < g.nx && j < g.ny && k < g.nz)
    acc = ((double)u[pidx(k, j, i, g.ny, g.nx)] + (g.ubase_d ? g.ubase_d[k] : 0.0)) * dzf[k];
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    partials[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
}

__global__ void k_bulk_finalize(const double* __restrict__ partials, int n, double* __restrict__ scal,
                                double scale, double U_target, double dt, int update_forcing) {
  __shared__ double sh[32];
  bulk_reduce_block(partials, n, scal, scale, U_target, dt, update_forcing, sh);
}

// ---------------------------------------------------------------------------
// CFL inverse time scale (operators.py:1232-1333): per-block maxima.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_cfl_partials(Grid<T> g, const T* __restrict__ u, const T* __restrict__ v,
                                                      const T* __restrict__ w, double* __restrict__ partials) {
  __shared__ double sh[32];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  double m = 0.0;
  if (i < nx && j < ny && k < nz) {
    const double top = g.top_neumann ? 1.0 : -1.0;
    Acc<T> U{u, nx, ny, nz, (T)top, g.ubase_t}, V{v, nx, ny, nz, (T)top, nullptr}, W{w, nx, ny, nz, (T)top, nullptr};
    const int im = wrap(i - 1, nx), ip = wrap(i + 1, nx), jm = wrap(j - 1, ny), jp = wrap(j + 1, ny);
    const double idx = (double)g.idx, idy = (double)g.idy, idzf = (double)g.idzf[k];
    double ux = fabs((double)U.c(k, j, i));
    double vx = 0.25 * fabs((double)V.c(k, j, i) + (double)V.c(k, jm, i) + (double)V.c(k, j, ip) + (double)V.c(k, jm, ip));
    double wx = 0.25 * fabs((double)W.f(k + 1, j, i) + (double)W.f(k, j, i) + (double)W.f(k + 1, j, ip) + (double)W.f(k, j, ip));
    m = ux * idx + vx * idy + wx * idzf;
    double uy = 0.25 * fabs((double)U.c(k, j, i) + (double)U.c(k, jp, i) + (double)U.c(k, jp, im) + (double)U.c(k, j, im));
    double vy = fabs((double)V.c(k, j, i));
    double wy = 0.25 * fabs((double)W.f(k + 1, j, i) + (double)W.f(k + 1, jp, i) + (double)W.f(k, jp, i) + (double)W.f(k, j, i));
    m = fmax(m, uy * idx + vy * idy + wy * idzf);
    if (k < nz - 1) {
      double uz = 0.25 * fabs((double)U.c(k, j, i) + (double)U.c(k, j, im) + (double)U.c(k + 1, j, im) + (double)U.c(k + 1, j, i));
      double vz = 0.25 * fabs((double)V.c(k, j, i) + (double)V.c(k, jm, i) + (double)V.c(k + 1, jm, i) + (double)V.c(k + 1, j, i));
      double wz = fabs((double)W.f(k + 1, j, i));
      m = fmax(m, uz * idx + vz * idy + wz * (double)g.idzc[k + 1]);
    }
  }
  double r = block_max(m, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    partials[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = r;
}

__global__ void k_max_finalize(const double* __restrict__ partials, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double m = 0.0;
  for (int e = threadIdx.x; e < n; e += blockDim.x) m = fmax(m, partials[e]);
  double r = block_max(m, sh);
  if (threadIdx.x == 0) *out = r;
}

// ---------------------------------------------------------------------------
// Diagnostics: max |div| (utils.py:226-240), non-finite scan of u, v, w, p
// (solver.py:865-868) -> per-block partials (max, flag).  The base profile of
// u cancels in the x difference.
// ---------------------------------------------------------------------------
template <class T, class PT = double>
__global__ void __launch_bounds__(256) k_diag_partials(Grid<T> g, const T* __restrict__ u, const T* __restrict__ v,
                                                       const T* __restrict__ w, const PT* __restrict__ p,
                                                       double* __restrict__ pmax, double* __restrict__ pflag) {
  __shared__ double sh[32];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  double m = 0.0, bad = 0.0;
  if (i < nx && j < ny && k < nz) {
    const size_t o = pidx(k, j, i, ny, nx);
    double du = ((double)u[o] - (double)u[pidx(k, j, wrap(i - 1, nx), ny, nx)]) * (double)g.idx;
    double dv = ((double)v[o] - (double)v[pidx(k, wrap(j - 1, ny), i, ny, nx)]) * (double)g.idy;
    double dw = ((double)w[pidx(k + 1, j, i, ny, nx)] - (double)w[o]) * (double)g.idzf[k];
    m = fabs(du + dv + dw);
    double s = (double)u[o] + (double)v[o] + (double)w[pidx(k + 1, j, i, ny, nx)] + (double)p[o];
    if (!isfinite(s)) bad = 1.0;
    if (!isfinite(m)) m = INFINITY;
  }
  double r = block_max(m, sh);
  double b = block_max(bad, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    size_t bi = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    pmax[bi] = r;
    pflag[bi] = b;
  }
}

// Ghost-inclusive plane sum of u (utils.py:187,201 take torch.mean over the
// whole (nx+1, ny+2) plane, periodic copies included): weights count how many
// reference entries alias each DOF.  One block per plane (bot, top).
template <class T>
__global__ void k_utau_sums(Grid<T> g, const T* __restrict__ u, double* __restrict__ scal) {
  __shared__ double sh[32];
  const int nx = g.nx, ny = g.ny;
  const int k = blockIdx.x == 0 ? 0 : g.nz - 1;
  const double bk = g.ubase_d ? g.ubase_d[k] : 0.0;
  double acc = 0.0;
  for (int e = threadIdx.x; e < nx * ny; e += blockDim.x) {
    int j = e / nx, i = e - j * nx;
    double wgt = (i == nx - 1 ? 2.0 : 1.0) * (1.0 + (j == 0 ? 1.0 : 0.0) + (j == ny - 1 ? 1.0 : 0.0));
    acc += wgt * ((double)u[pidx(k, j, i, ny, nx)] + bk);
  }
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0) scal[SC_UTAU_BOT + blockIdx.x] = s / ((double)(nx + 1) * (double)(ny + 2));
}

// ---------------------------------------------------------------------------
// Reference layout <-> internal layout.
// Reference arrays are C order (X, Y, Z) with Z fastest.  A 32x32 tile over
// (x, z) for a fixed y row is staged through shared memory so both sides
// coalesce.
// ---------------------------------------------------------------------------
enum : int { FLD_U = 0, FLD_V = 1, FLD_W = 2, FLD_P = 3, FLD_CELL = 4 };

// Gather the DOFs of a reference array into the internal layout.
// FLD_U/V: ref (Xr, Yr, nz+2) -> internal [nz][ny][nx] = ref[i+1, j+1, k+1] - base[k]
// FLD_W:   ref (nx+2, ny+2, nz+1) -> internal [nz+1][ny][nx] = ref[i+1, j+1, k]
//          (wall planes written as 0)
// FLD_CELL: ref (nx, ny, nz) -> internal [nz][ny][nx] = ref[i, j, k] * scale
template <class T>
__global__ void k_from_ref(const double* __restrict__ ref, T* __restrict__ out, int kind, int nx, int ny, int nz,
                           double scale, const double* __restrict__ base) {
  __shared__ double tile[32][33];
  const int j = blockIdx.y;
  const int i0 = blockIdx.x * 32, k0 = blockIdx.z * 32;
  int Yr, Zr, ox, oy, oz, NK;
  switch (kind) {
    case FLD_U: Yr = ny + 2; Zr = nz + 2; ox = 1; oy = 1; oz = 1; NK = nz; break;
    case FLD_V: Yr = ny + 1; Zr = nz + 2; ox = 1; oy = 1; oz = 1; NK = nz; break;
    case FLD_W: Yr = ny + 2; Zr = nz + 1; ox = 1; oy = 1; oz = 0; NK = nz + 1; break;
    default: Yr = ny; Zr = nz; ox = 0; oy = 0; oz = 0; NK = nz; break;
  }
  // read: threadIdx.x along z (contiguous in ref)
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int i = i0 + r, k = k0 + threadIdx.x;
    double val = 0.0;
    if (i < nx && k < NK) val = ref[((size_t)(i + ox) * Yr + (j + oy)) * Zr + (k + oz)] * scale;
    tile[r][threadIdx.x] = val;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int k = k0 + r, i = i0 + threadIdx.x;
    if (i < nx && k < NK) {
      double val = tile[threadIdx.x][r];
      if (kind == FLD_W && (k == 0 || k == nz)) val = 0.0;
      if (base) val -= base[k];
      out[pidx(k, j, i, ny, nx)] = (T)val;
    }
  }
}

// Per-plane mean of the DOFs of a reference u array: the base profile of the
// mixed-precision storage.  One block per plane.
__global__ void k_plane_mean_ref_u(const double* __restrict__ ref, int nx, int ny, int nz, double* __restrict__ out) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  double acc = 0.0;
  for (int e = threadIdx.x; e < nx * ny; e += blockDim.x) {
    int i = e / ny, j = e - i * ny;
    acc += ref[((size_t)(i + 1) * (ny + 2) + (j + 1)) * (nz + 2) + (k + 1)];
  }
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0) out[k] = s / ((double)nx * (double)ny);
}

// Materialise a full reference array (ghosts included) from the internal
// layout, with the ghost rules of apply_bc_all (solver.py:23-79) and of the
// pressure ghost fill (projection_fft.py:148-163).  `base` (u only) is added
// back to the stored values.
template <class T>
__global__ void k_to_ref(const T* __restrict__ in, double* __restrict__ ref, int kind, int nx, int ny, int nz,
                         int top_neumann, const double* __restrict__ base) {
  __shared__ double tile[32][33];
  int Xr, Yr, Zr;
  switch (kind) {
    case FLD_U: Xr = nx + 1; Yr = ny + 2; Zr = nz + 2; break;
    case FLD_V: Xr = nx + 2; Yr = ny + 1; Zr = nz + 2; break;
    case FLD_W: Xr = nx + 2; Yr = ny + 2; Zr = nz + 1; break;
    case FLD_P: Xr = nx + 2; Yr = ny + 2; Zr = nz + 2; break;
    default: Xr = nx; Yr = ny; Zr = nz; break;
  }
  const int J = blockIdx.y;
  const int I0 = blockIdx.x * 32, K0 = blockIdx.z * 32;
  // internal row index for J
  int j;
  if (kind == FLD_CELL) j = J;
  else if (kind == FLD_V) j = (J == 0) ? ny - 1 : J - 1;
  else j = (J == 0) ? ny - 1 : (J == ny + 1 ? 0 : J - 1);
  const double top = top_neumann ? 1.0 : -1.0;
  // read internal: threadIdx.x along x
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int K = K0 + r, I = I0 + threadIdx.x;
    double val = 0.0;
    if (I < Xr && K < Zr) {
      int i;
      if (kind == FLD_CELL) i = I;
      else if (kind == FLD_U) i = (I == 0) ? nx - 1 : I - 1;
      else i = (I == 0) ? nx - 1 : (I == nx + 1 ? 0 : I - 1);
      if (kind == FLD_W || kind == FLD_CELL) {
        val = (double)in[pidx(K, j, i, ny, nx)];
      } else if (kind == FLD_P) {
        int k = K == 0 ? 0 : (K == nz + 1 ? nz - 1 : K - 1);
        val = (double)in[pidx(k, j, i, ny, nx)];
      } else {
        auto tot = [&](int k) { return (double)in[pidx(k, j, i, ny, nx)] + (base ? base[k] : 0.0); };
        if (K == 0) val = -tot(0);
        else if (K == nz + 1) val = top * tot(nz - 1);
        else val = tot(K - 1);
      }
    }
    tile[r][threadIdx.x] = val;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int I = I0 + r, K = K0 + threadIdx.x;
    if (I < Xr && K < Zr) ref[((size_t)I * Yr + J) * Zr + K] = tile[threadIdx.x][r];
  }
}

}  // namespace tc
