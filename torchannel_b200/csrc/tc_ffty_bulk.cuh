// FFT along y of the rows X[kx][k][:] of the Poisson spectrum (kernel c,
// projection_fft.py:117-139) with the rows staged in shared memory by bulk
// copies of the tensor memory accelerator instead of per-lane loads.
//
// A tile is R = 4 RowFft::RPW consecutive rows of X (one contiguous run of
// R N complex values).  Persistent CTAs of four warps walk the tiles with two
// stages: while the warps transform the rows of one stage in place, the bulk
// copies of the next tile's rows land in the other, and the transformed rows
// leave by bulk stores.  A row's transpose tile overlays the row itself (the
// warp reads the row into registers first), so a stage row holds
// RowFft::TILE >= N complex values.  The arithmetic is that of k_ffty_reg
// (rowfft_pass1_regs, then the N2-point DFTs of pass 2), so the results are
// the same bits; only the staging differs: no load or store instruction of
// the lanes touches global memory, which leaves the issue slots to the
// transforms.
// Each wait on a stage's barrier is bounded; if one runs out, the CTA sets
// TCE_TIMEOUT in the error word, waits (bounded) for its own copies in flight
// and returns.
#pragma once
#include "tc_async.cuh"
#include "tc_fft_reg.cuh"
#undef TC_FILE_ID
#define TC_FILE_ID 4

namespace tc {

template <int N1> struct YBulk {
  using RF = RowFft<N1>;
  static constexpr int N = RF::N;
  static constexpr int NW = 4;                       // warps per CTA
  static constexpr int R = NW * RF::RPW;             // rows per tile
  static constexpr int SP = (RF::TILE + 7) / 8 * 8;  // stage row pitch (complex): the row or its transpose tile
  static constexpr int NST = 2;                      // stages
  static constexpr size_t STAGE = (size_t)R * SP * sizeof(cpx<double>);
  static constexpr unsigned ROW_BYTES = (unsigned)(N * sizeof(cpx<double>));
  static_assert(ROW_BYTES % 16 == 0 && (SP * sizeof(cpx<double>)) % 128 == 0, "bulk-copy alignment");
  static __host__ __device__ constexpr size_t smem() { return NST * STAGE + NST * 8; }
  // resident CTAs per SM the registers are bounded for (longer rows need more)
  static constexpr int MINB = N1 <= 8 ? 4 : (N1 <= 18 ? 3 : 2);
};

#define YBULK_WAIT_LIMIT (1u << 21)

template <int N1, bool INV>
__global__ void __launch_bounds__(128, YBulk<N1>::MINB) k_ffty_bulk(cpx<double>* __restrict__ X, int nrows,
                                                      const cpx<double>* __restrict__ twy, int* __restrict__ err) {
  using B = YBulk<N1>;
  using RF = typename B::RF;
  constexpr int N = B::N, R = B::R, SP = B::SP;
  extern __shared__ __align__(16) unsigned char smraw[];  // 128-byte alignment checked below
  cpx<double>* stages = reinterpret_cast<cpx<double>*>(smraw);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw + B::NST * B::STAGE);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int sub = lane / RF::LANES, l = lane - sub * RF::LANES;
  const int wr = warp * RF::RPW + sub;  // the lane's row of a tile
  const bool rl = sub < RF::RPW;
  const int ntiles = (nrows + R - 1) / R;
  if (blockIdx.x >= ntiles) return;
  if (smem_u32(smraw) & 127u) {  // bulk copies need aligned rows
    if (tid == 0) atomicOr(err, TCE_BOUNDS);
    return;
  }
  if (tid == 0) {
    for (int q = 0; q < B::NST; ++q) mbar_init(&bar[q], 1);
    mbar_init_fence();
  }
  __syncthreads();
  // rows of tile t that exist (and, in bounds-checked builds, pass the check)
  auto tile_rows = [&](int t) {
    const int r0 = t * R, nr = min(R, nrows - r0);
    int ok = 0;
    for (int r = 0; r < nr; ++r) ok += TC_IN((size_t)(r0 + r) * N, (size_t)nrows * N, N) ? 1 : 0;
    return ok == nr ? nr : 0;
  };
  auto issue = [&](int t, int s) {  // one thread
    const int r0 = t * R, nr = tile_rows(t);
    cpx<double>* st = stages + (size_t)s * R * SP;
    mbar_expect_tx(&bar[s], (unsigned)nr * B::ROW_BYTES);
    for (int r = 0; r < nr; ++r) bulk_load(st + (size_t)r * SP, X + (size_t)(r0 + r) * N, B::ROW_BYTES, &bar[s]);
  };
  if (tid == 0) issue(blockIdx.x, 0);
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int s = it & 1;
    const int tn = t + (int)gridDim.x;
    if (tid == 0) {
      bulk_wait_read();  // the last tile's stores (stage s ^ 1) have read their rows
      if (tn < ntiles) issue(tn, s ^ 1);
    }
    const bool landed = mbar_wait_bounded(&bar[s], (unsigned)(it >> 1) & 1u, YBULK_WAIT_LIMIT);
    if (__syncthreads_or(!landed)) {
      if (tid == 0) {
        // let the copies in flight land (bounded) before the CTA leaves
        mbar_wait_bounded(&bar[s], (unsigned)(it >> 1) & 1u, YBULK_WAIT_LIMIT);
        if (tn < ntiles) mbar_wait_bounded(&bar[s ^ 1], (unsigned)((it + 1) >> 1) & 1u, YBULK_WAIT_LIMIT);
        bulk_wait_all();
        atomicOr(err, TCE_TIMEOUT);
      }
      return;
    }
    const int r0 = t * R, nr = tile_rows(t);
    cpx<double>* row = stages + (size_t)s * R * SP + (size_t)(rl ? wr : 0) * SP;
    const bool ok = rl && wr < nr;
    cpx<double> v[RF::N1];
    if (ok && l < RF::N2) {
#pragma unroll
      for (int n1 = 0; n1 < RF::N1; ++n1) v[n1] = row[RF::N2 * n1 + l];
    }
    __syncwarp();
    if (ok && l < RF::N2) rowfft_pass1_regs<N1, INV>(v, l, row, twy);  // the transpose tile overlays the row
    __syncwarp();
    cpx<double> b[RF::N2];
    if (ok && l < RF::N1) {
#pragma unroll
      for (int n2 = 0; n2 < RF::N2; ++n2) b[n2] = row[l * RF::TP + n2];
    }
    __syncwarp();
    if (ok && l < RF::N1) {
      Dft<RF::N2, INV>::run(b);
#pragma unroll
      for (int k2 = 0; k2 < RF::N2; ++k2) row[l + RF::N1 * k2] = b[k2];  // the row, natural order
    }
    bulk_store_fence();
    __syncthreads();
    if (tid == 0) {
      const cpx<double>* st = stages + (size_t)s * R * SP;
      for (int r = 0; r < nr; ++r) bulk_store(X + (size_t)(r0 + r) * N, st + (size_t)r * SP, B::ROW_BYTES);
      bulk_commit();
    }
  }
  if (tid == 0) bulk_wait_all();
}

}  // namespace tc
