// Kernel (a) with its tiles staged by the tensor memory accelerator: the
// stencils of rhs_stencils (advection + x/y or full diffusion + forcing + AB2,
// operators.py:18-248, 474-548, 818-1225; solver.py:626-651) over tiles of
// RHS_TX x 8 points and KB planes, in a persistent loop of CTAs that each
// hold two stages in shared memory.  While a CTA evaluates one tile, one
// thread has already issued the 3-D tensor copies (cp.async.bulk.tensor) of
// the u, v and w boxes of its next tile into the other stage, so that the
// staging costs no load or store instructions and its latency hides behind
// the arithmetic.
//
// Box of a tile (i0, j0, kb): x from i0 - XA (XA = 16 bytes / sizeof(T), so
// that the copy starts on a 16-byte boundary) over RHS_TX + 2 XA columns, y
// from j0 - 1 over 10 rows, planes kb - 1 .. kb + KB.  What the box cannot
// hold is patched after it lands:
//  * periodic wraps (tiles at the x / y ends of the domain): the halo
//    column / row from the other end, loaded from global memory;
//  * u / v z ghosts (planes -1 and nz, which the box reads as zeros):
//    -q[0] below, -q[nz-1] (no-slip) or +q[nz-1] (free-slip) above; w's
//    plane -1 stays 0 and its plane nz is the stored wall;
//  * mixed precision: u is stored as u - U0[k]; the stencils add U0[k] to
//    their sums of u (rhs_march).
// Each wait on a stage's barrier is bounded; if one runs out, the CTA sets
// TCE_TIMEOUT in the error word and stops.
#pragma once
#include "tc_async.cuh"
#include "tc_step.cuh"
#undef TC_FILE_ID
#define TC_FILE_ID 2

namespace tc {

template <class T, int KB, int NST = 2> struct RhsTma {
  static constexpr int XA = 16 / (int)sizeof(T);  // x alignment of a box start (elements)
  static constexpr int BX = RHS_TX + 2 * XA;      // box columns: x = i0 - XA ..
  static constexpr int OX = XA;                   // box column of x = i0
  static constexpr int TY = 8;                    // rows of a tile
  static constexpr int BY = TY + 2;               // box rows: y = j0 - 1 ..
  static constexpr int BZ = KB + 2;               // box planes: kb - 1 .. kb + KB
  static constexpr int BOX = BX * BY * BZ;        // elements of one field's box
  static constexpr int STAGE = 3 * BOX;           // u, v, w
  static constexpr unsigned BOX_BYTES = (unsigned)(BOX * sizeof(T));
  static_assert(BOX_BYTES % 128 == 0, "boxes must stay 128-byte aligned in shared memory");
  // stages, two mbarriers, the march's per-tile constants (rhs_pre_value)
  static constexpr int PRE = rhs_pre_count<T, KB>();
  static __host__ __device__ constexpr size_t smem() { return NST * (size_t)STAGE * sizeof(T) + 2 * 8 + PRE * sizeof(T); }
};

#define RHS_TMA_WAIT_LIMIT (1u << 21)

// Issue the tensor copies of tile (bx, by, bz) into stage d, completing on
// bar (one thread; the maps are addresses of __grid_constant__ parameters).
template <class T, int KB, int NST>
__device__ __forceinline__ void rhs_tma_issue(T* d, uint64_t* bar, const CUtensorMap* mu, const CUtensorMap* mv,
                                              const CUtensorMap* mw, int bx, int by, int bz) {
  using S = RhsTma<T, KB, NST>;
  mbar_expect_tx(bar, 3 * S::BOX_BYTES);
  const int x = bx * RHS_TX - S::XA, y = by * S::TY - 1, z = bz * KB - 1;
  tma_load_3d(d, mu, x, y, z, bar);
  tma_load_3d(d + S::BOX, mv, x, y, z, bar);
  tma_load_3d(d + 2 * S::BOX, mw, x, y, z, bar);
}

// One tile (bx, by, bz) whose copies into `stage` were issued on `bar`
// (phase `par`): the loads that do not need the copy (AB2 history, the
// march's per-tile constants into `pre`, the periodic-wrap patch), the
// bounded wait, the patches and the stencils.  False when the wait ran out:
// the CTA has set TCE_TIMEOUT in `err` and let its copies in flight land
// (bounded; `bar_other` / `par_other`: a second stage with a copy in flight,
// or nullptr), and must leave without further barriers.
template <class T, bool FULL, int UPD, int KB, int NST>
__device__ __forceinline__ bool rhs_tma_tile(const Grid<T>& g, const T* __restrict__ u, const T* __restrict__ v,
                                             const T* __restrict__ w, T* __restrict__ us, T* __restrict__ vs,
                                             T* __restrict__ ws, T* __restrict__ ru, T* __restrict__ rv,
                                             T* __restrict__ rw, T forcing, T dt, int have_hist, int bx, int by,
                                             int bz, T* stage, uint64_t* bar, unsigned par, T* pre, int* err,
                                             uint64_t* bar_other, unsigned par_other) {
  using S = RhsTma<T, KB, NST>;
  constexpr int BX = S::BX, BY = S::BY, BZ = S::BZ, OX = S::OX;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const size_t plane = (size_t)nx * ny;
  const size_t ncell = plane * nz, nface = plane * (nz + 1);  // field extents (bounds-checked builds)
  (void)ncell; (void)nface;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * RHS_TX + tx, nthr = RHS_TX * S::TY;
  const T top = g.top_neumann ? T(1) : T(-1);
  const int i0 = bx * RHS_TX, j0 = by * S::TY, kb = bz * KB;
  const int i = i0 + tx, j = j0 + ty;
  const bool active = (i < nx) && (j < ny);
  // AB2 history of this thread's points, in flight with the copy
  T hru[KB], hrv[KB], hrw[KB];
#pragma unroll
  for (int q = 0; q < KB; ++q) {
    const int k = kb + q;
    const unsigned o = (unsigned)k * (unsigned)plane + (unsigned)j * (unsigned)nx + (unsigned)i;  // < 2^32
    const bool cell = active && k < nz, face = active && k >= 1 && k <= nz - 1;
    const bool hist = UPD == UPD_AB2 && have_hist;
    hru[q] = (cell && hist && TC_IN(o, ncell, 1)) ? ru[o] : T(0);
    hrv[q] = (cell && hist && TC_IN(o, ncell, 1)) ? rv[o] : T(0);
    hrw[q] = (face && hist && TC_IN(o, nface, 1)) ? rw[o] : T(0);
  }
  // the march's per-tile constants (the last tile's were read before the
  // barrier that ended it)
  if (sizeof(T) == 4 && tid < S::PRE) pre[tid] = rhs_pre_value<T, KB>(g, kb, tid);
  // periodic wraps of the halo ring (tiles at the x / y ends of the domain):
  // ring positions of a plane are 2 columns of BY rows and 2 rows of
  // RHS_TX + 2; entry e of the box's ring gives its box index and, when it
  // lies outside the domain, the wrapped offset in the plane.  The loads
  // of the thread's first WR entries are in flight with the copy.
  constexpr int RING = 2 * BY + 2 * (RHS_TX + 2), NRING = RING * BZ, WR = 4;
  const bool wrap_x = (i0 == 0) || (i0 + RHS_TX >= nx);
  const bool wrap_y = (j0 == 0) || (j0 + S::TY >= ny);
  const bool wrap_tile = wrap_x || wrap_y;
  auto ring_entry = [&](int e, int& sidx, size_t& off) -> bool {
    const int sl = e / RING, q = e - sl * RING;
    int hy, hx;  // box row, and box column relative to x = i0 - 1
    if (q < 2 * BY) {
      hy = q % BY;
      hx = (q < BY) ? 0 : min(nx - i0, RHS_TX) + 1;
    } else {
      const int r = q - 2 * BY;
      hx = r % (RHS_TX + 2);
      hy = (r < RHS_TX + 2) ? 0 : min(ny - j0, S::TY) + 1;
    }
    const int xg = i0 - 1 + hx, yg = j0 - 1 + hy;
    if (xg >= 0 && xg < nx && yg >= 0 && yg < ny) return false;  // inside the domain: the box holds it
    off = (size_t)(kb - 1 + sl) * plane + (size_t)wrap(yg, ny) * nx + wrap(xg, nx);
    sidx = (sl * BY + hy) * BX + OX - 1 + hx;
    return true;
  };
  // plane of a ring entry's box index: slot sl = sidx / (BY BX) is plane kb-1+sl
  auto ring_plane = [&](int sidx) { return kb - 1 + sidx / (BY * BX); };
  T wu[WR], wv[WR], ww[WR];
  int wsi[WR];
#pragma unroll
  for (int r = 0; r < WR; ++r) {
    const int e = tid + r * nthr;
    int sidx = -1;
    size_t off = 0;
    wu[r] = wv[r] = ww[r] = T(0);
    if (wrap_tile && e < NRING && ring_entry(e, sidx, off)) {
      const int p = ring_plane(sidx);
      if (p >= 0 && p < nz && TC_IN(off, ncell, 1)) {
        wu[r] = ldg(u + off);
        wv[r] = ldg(v + off);
      }
      if (p >= 0 && p <= nz && TC_IN(off, nface, 1)) ww[r] = ldg(w + off);
    } else {
      sidx = -1;
    }
    wsi[r] = sidx;
  }
  const bool landed = mbar_wait_bounded(bar, par, RHS_TMA_WAIT_LIMIT);
  if (__syncthreads_or(!landed)) {
    if (tid == 0) {
      // let the copies in flight finish (bounded) before leaving
      mbar_wait_bounded(bar, par, RHS_TMA_WAIT_LIMIT);
      if (bar_other) mbar_wait_bounded(bar_other, par_other, RHS_TMA_WAIT_LIMIT);
      atomicOr(err, TCE_TIMEOUT);
    }
    return false;
  }
  T* su = stage;
  T* sv = su + S::BOX;
  T* sw = sv + S::BOX;
  // (1) periodic wraps of the halo ring (stored values) on the planes that
  //     exist: the entries loaded before the copy landed, then the rest
  if (wrap_tile) {
#pragma unroll
    for (int r = 0; r < WR; ++r) {
      const int sidx = wsi[r];
      if (sidx < 0) continue;
      const int p = ring_plane(sidx);
      if (p >= 0 && p < nz) {
        su[sidx] = wu[r];
        sv[sidx] = wv[r];
      }
      if (p >= 0 && p <= nz) sw[sidx] = ww[r];
    }
    for (int e = tid + WR * nthr; e < NRING; e += nthr) {
      int sidx;
      size_t off;
      if (!ring_entry(e, sidx, off)) continue;
      const int p = ring_plane(sidx);
      if (p >= 0 && p < nz && TC_IN(off, ncell, 1)) {
        su[sidx] = ldg(u + off);
        sv[sidx] = ldg(v + off);
      }
      if (p >= 0 && p <= nz && TC_IN(off, nface, 1)) sw[sidx] = ldg(w + off);
    }
    __syncthreads();
  }
  // (2) z ghosts of u and v: plane -1 (slot 0 of the first tile) and plane
  //     nz (slot nz - kb + 1 when it is in the box)
  const int sg_lo = (kb == 0) ? 0 : -1;
  const int sg_hi = (nz - kb + 1 < BZ) ? nz - kb + 1 : -1;
  if (sg_lo >= 0 || sg_hi >= 0) {
    for (int e = tid; e < 2 * BY * (RHS_TX + 2); e += nthr) {
      const int which = e / (BY * (RHS_TX + 2)), r = e - which * (BY * (RHS_TX + 2));
      const int hy = r / (RHS_TX + 2), hx = r - hy * (RHS_TX + 2);
      const int sl = which == 0 ? sg_lo : sg_hi;
      if (sl < 0) continue;
      const int from = which == 0 ? sl + 1 : sl - 1;
      const T sgn = which == 0 ? T(-1) : top;
      const int a = (sl * BY + hy) * BX + OX - 1 + hx, b = (from * BY + hy) * BX + OX - 1 + hx;
      su[a] = sgn * su[b];
      sv[a] = sgn * sv[b];
    }
    __syncthreads();
  }
  // (3) the stencils, marching up the thread's column (as in rhs_tile)
  rhs_stencils<T, FULL, UPD, KB, BY, BX>(g, reinterpret_cast<const T(*)[BY][BX]>(su),
                                         reinterpret_cast<const T(*)[BY][BX]>(sv),
                                         reinterpret_cast<const T(*)[BY][BX]>(sw), tx + OX, ty + 1, i, j, active,
                                         kb, us, vs, ws, ru, rv, rw, hru, hrv, hrw, forcing, dt, have_hist,
                                         sizeof(T) == 4 ? pre : nullptr);
  return true;
}

// NST stages: 2 = a persistent pipeline (the next tile's copy in flight
// while this one is evaluated), 1 = one tile per CTA (latency hidden by the
// other resident CTAs); MINB = resident CTAs per SM the registers allow.
template <class T, bool FULL, int UPD, int KB, int NST, int MINB>
__global__ void __launch_bounds__(RHS_TX * 8, MINB)
    k_rhs_tma(const __grid_constant__ CUtensorMap mu, const __grid_constant__ CUtensorMap mv,
              const __grid_constant__ CUtensorMap mw, Grid<T> g, const T* __restrict__ u, const T* __restrict__ v,
              const T* __restrict__ w, T* __restrict__ us, T* __restrict__ vs, T* __restrict__ ws,
              T* __restrict__ ru, T* __restrict__ rv, T* __restrict__ rw, const double* __restrict__ forcing_dev,
              T dt, int have_hist, int ntx, int nty, int ntz, int* __restrict__ err) {
  using S = RhsTma<T, KB, NST>;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* buf = reinterpret_cast<T*>(smraw);
  uint64_t* bar = reinterpret_cast<uint64_t*>(buf + NST * S::STAGE);
  T* pre = reinterpret_cast<T*>(bar + 2);
  const int tid = threadIdx.y * RHS_TX + threadIdx.x;
  const int ntiles = ntx * nty * ntz;
  const T forcing = (UPD == UPD_AB2) ? (T)(*forcing_dev) : T(0);
  if (blockIdx.x >= ntiles) return;
  if (smem_u32(buf) & 127u) {  // tensor copies need 128-byte aligned boxes
    if (tid == 0) atomicOr(err, TCE_BOUNDS);
    return;
  }
  if (tid == 0) {
    tma_prefetch_desc(&mu);
    tma_prefetch_desc(&mv);
    tma_prefetch_desc(&mw);
    for (int q = 0; q < NST; ++q) mbar_init(&bar[q], 1);
    mbar_init_fence();
  }
  __syncthreads();
  auto decode = [&](int t, int& bx, int& by, int& bz) {
    bz = t % ntz;
    const int r = t / ntz;
    by = r % nty;
    bx = r / nty;
  };
  auto issue = [&](int t, int st) {  // one thread
    int bx, by, bz;
    decode(t, bx, by, bz);
    rhs_tma_issue<T, KB, NST>(buf + (size_t)st * S::STAGE, &bar[st], &mu, &mv, &mw, bx, by, bz);
  };
  if (tid == 0) issue(blockIdx.x, 0);
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int st = NST == 2 ? (it & 1) : 0;
    const unsigned par = NST == 2 ? (unsigned)(it >> 1) & 1u : (unsigned)it & 1u;
    // the other stage was released by the barrier that ended the last tile;
    // with one stage the next copy waits for this tile's end
    const bool next2 = NST == 2 && t + (int)gridDim.x < ntiles;
    if (next2 && tid == 0) issue(t + gridDim.x, st ^ 1);
    int bx, by, bz;
    decode(t, bx, by, bz);
    if (!rhs_tma_tile<T, FULL, UPD, KB, NST>(g, u, v, w, us, vs, ws, ru, rv, rw, forcing, dt, have_hist, bx, by, bz,
                                             buf + (size_t)st * S::STAGE, &bar[st], par, pre, err,
                                             next2 ? &bar[st ^ 1] : nullptr, (unsigned)((it + 1) >> 1) & 1u))
      return;
    __syncthreads();  // this stage is free for the copy issued two tiles on
    if (NST == 1 && tid == 0 && t + (int)gridDim.x < ntiles) issue(t + gridDim.x, 0);
  }
}

// Tiles of k_rhs_tma: x tiles, y tiles, z tiles of KB planes (planes 0 .. nz-1).
__host__ inline void rhs_tma_tiles(int nx, int ny, int nz, int kb, int* ntx, int* nty, int* ntz) {
  *ntx = (nx + RHS_TX - 1) / RHS_TX;
  *nty = (ny + 7) / 8;
  *ntz = (nz + kb - 1) / kb;
}

}  // namespace tc
