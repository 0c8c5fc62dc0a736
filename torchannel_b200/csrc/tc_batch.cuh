// Ensemble kernels: one persistent launch per substep for every member of an
// ensemble of independent channels with uneven grids.
//
// A launch's work is the concatenation of the members' work units (the
// blocks -- or, for the y transforms, the warp tasks -- each member's own
// kernel would run); member m owns units [BMember::u0[K], u0[K] + count).  A
// fixed grid of CTAs (a multiple of the SM count) strides over the units, so
// the launch is persistent and small members fill the SMs together.  Each unit
// runs the same tile function as the single-channel kernel (rhs_tile,
// cn_tile, fftx_tile, ffty_rows, tri_lu2_thread, ifftx_tile, project_tile), so
// a member's results are bit-identical to stepping it alone with the same
// CN chunk length.  Units that share the block's shared memory are separated
// by a barrier.
#pragma once
#include "tc_common.cuh"
#include "tc_poisson.cuh"
#include "tc_rhs_tma.cuh"
#include "tc_step.cuh"

namespace tc {

enum : int { BK_RHS = 0, BK_CN, BK_FX, BK_FY, BK_TRI, BK_IFX, BK_PROJ, BK_COUNT };
#define TC_BATCH_MAX 64  // members per ensemble launch

// Register allocation of the unit loops.  The x transforms run one launch
// per transform length (kb_fftx_n, kb_ifftx_n: the registers of that length
// alone, where one kernel over all lengths takes those of the longest and
// spills), one CTA per unit: TC_BATCH_XP planes of a row block (forward) or
// one plane (inverse).  A persistent unit loop around the same tiles took
// 128-192 registers and, capped at 96, spilled; the forward transform with
// one plane a CTA measured slower than with TC_BATCH_XP.  The other loops
// inline their tiles under occupancy-driven register caps (minimum resident
// blocks per SM below).
#ifndef TC_BATCH_FFT_MINB
#define TC_BATCH_FFT_MINB 4
#endif
#ifndef TC_BATCH_RHS_MINB
#define TC_BATCH_RHS_MINB 6      // FP64 storage (the per-plane stencils)
#endif
#ifndef TC_BATCH_RHS_MINB32
#define TC_BATCH_RHS_MINB32 3    // FP32 storage (the column march carries plane values: 80 registers)
#endif
#ifndef TC_BATCH_XP
#define TC_BATCH_XP 4
#endif

template <class T> struct BMember {
  Grid<T> g;
  T* A[3];                 // state at the start of the step
  T* B[3];                 // u*, then u**, then the new state
  T* R[3];                 // AB2 history
  const double* forcing;   // device forcing scalar of the member
  T dt;
  int have_hist;
  CnTab tab;
  const double* ubase;     // FP64 base profile of u (mixed) or null
  cpx<double>* X;
  const cpx<double>* twx;
  const cpx<double>* twy;
  double scale;            // 1 / (dt nx ny)
  const double* rden;
  const double* cpt;
  PoissonTabs tb;
  double* p;
  const double* dzf;
  BulkArgs ba;
  int n1y, nxh, nrows;
  int rgx, rgy, rgz;       // block grid of k_rhs_update
  int tnx, tny, tnz;       // tiles of the tensor-copy RHS (k_rhs_tma's default shape)
  int cgx;                 // column blocks per component of k_cn_solve
  int xgx;                 // row blocks per plane of the x transforms
  int xpg;                 // plane groups of the forward x transform
  int pgx, pgy, pgz;       // block grid of k_project_bulk
  int u0[BK_COUNT];        // first unit of the member in each launch
};

// Member of a class launch owning unit w: the last k with st[k] <= w
// (binary search over the launch parameter's first units).
__device__ __forceinline__ int batch_class_member(const int* st, int n, int w) {
  int lo = 0, hi = n - 1;  // the last member whose first unit is <= w
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (st[mid] <= w) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Stage the members' first units of launch K (and the total) in shared memory.
template <class T>
__device__ __forceinline__ void batch_starts(const BMember<T>* __restrict__ M, int nm, int K, int total, int* st) {
  for (int m = threadIdx.x + blockDim.x * threadIdx.y; m < nm; m += blockDim.x * blockDim.y) st[m] = M[m].u0[K];
  if (threadIdx.x == 0 && threadIdx.y == 0) st[nm] = total;
  __syncthreads();
}

// Member owning unit w: the last m with st[m] <= w (binary search).
__device__ __forceinline__ int batch_member(const int* st, int nm, int w) {
  int lo = 0, hi = nm - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (st[mid] <= w) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <class T, bool FULL, int UPD>
__global__ void __launch_bounds__(RHS_TX * rhs_ty<T>(), sizeof(T) == 4 ? TC_BATCH_RHS_MINB32 : TC_BATCH_RHS_MINB) kb_rhs(const BMember<T>* __restrict__ M, int nm, int total) {
  __shared__ int st[TC_BATCH_MAX + 1];
  batch_starts(M, nm, BK_RHS, total, st);
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    const int m = batch_member(st, nm, w);
    const BMember<T>& b = M[m];
    int l = w - st[m];
    const int bx = l % b.rgx;
    l /= b.rgx;
    const int by = l % b.rgy, bz = l / b.rgy;
    rhs_tile<T, FULL, UPD>(b.g, b.A[0], b.A[1], b.A[2], b.B[0], b.B[1], b.B[2], b.R[0], b.R[1], b.R[2], b.forcing,
                           b.dt, UPD == UPD_FE ? 0 : b.have_hist, bx, by, bz);
    __syncthreads();
  }
}

// The explicit RHS of the members with their tiles staged by tensor copies
// (kb_rhs_tma).  Everything a tile reads of its member -- the tensor maps of
// u, v, w for the step's parity, the grid, the buffers, dt -- travels in the
// launch's __grid_constant__ parameter, as the single-channel kernel's does:
// the CTA's member is uniform, so its fields are uniform parameter loads and
// take no per-thread registers (read from a table in global memory they
// would, and spill).  A parameter holds TC_BATCH_TMA_GROUP members (within
// the 32,764-byte parameter limit); larger ensembles take one launch per
// group.
#define TC_BATCH_TMA_GROUP 32
template <class T> struct BRhsRec {
  Grid<T> g;
  T* A[3];
  T* B[3];
  T* R[3];
  const double* forcing;
  int* err;
  T dt;
  int have_hist;
  int tny, tnz;  // y and z tiles (z fastest)
};
template <class T> struct BatchRhsArgs {
  CUtensorMap map[TC_BATCH_TMA_GROUP][3];
  BRhsRec<T> r[TC_BATCH_TMA_GROUP];
  int st[TC_BATCH_TMA_GROUP + 1];  // first unit of each member of the group (global unit index), then the end
  int nm;
};
static_assert(sizeof(BatchRhsArgs<double>) + 64 <= 32764, "kernel parameter limit");

// Unit w = tile (bx, by, bz) of k_rhs_tma's default shape of its member,
// evaluated by the same tile code (rhs_tma_tile).  Persistent CTAs walk the
// group's units with one stage: the next unit's copies are issued once the
// barrier that ends a unit has released the stage (the other resident CTAs
// hide their latency, as for k_rhs_tma's one-tile CTAs).  Dynamic shared
// memory: the stage, its barrier and the march's constants.
template <class T> struct BatchRhsTmaShape {
  static constexpr int KB = sizeof(T) == 4 ? 8 : 2, MINB = sizeof(T) == 4 ? 3 : 5;
  using S = RhsTma<T, KB, 1>;
  static __host__ __device__ constexpr size_t smem() { return S::smem(); }
};
template <class T, bool FULL, int UPD>
__global__ void __launch_bounds__(RHS_TX * 8, BatchRhsTmaShape<T>::MINB)
    kb_rhs_tma(const __grid_constant__ BatchRhsArgs<T> a) {
  using B = BatchRhsTmaShape<T>;
  using S = typename B::S;
  constexpr int KB = B::KB;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* buf = reinterpret_cast<T*>(smraw);
  uint64_t* bar = reinterpret_cast<uint64_t*>(buf + S::STAGE);
  T* pre = reinterpret_cast<T*>(bar + 2);
  const int tid = threadIdx.y * RHS_TX + threadIdx.x;
  const int u0 = a.st[0], u1 = a.st[a.nm];
  if (u0 + (int)blockIdx.x >= u1) return;
  if (smem_u32(buf) & 127u) {  // tensor copies need 128-byte aligned boxes
    if (tid == 0) atomicOr(a.r[0].err, TCE_BOUNDS);
    return;
  }
  auto decode = [&](int w, int& m, int& bx, int& by, int& bz) {
    int lo = 0, hi = a.nm - 1;  // the last member whose first unit is <= w
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.st[mid] <= w) lo = mid; else hi = mid - 1;
    }
    m = lo;
    int l = w - a.st[m];
    bz = l % a.r[m].tnz;
    l /= a.r[m].tnz;
    by = l % a.r[m].tny;
    bx = l / a.r[m].tny;
  };
  auto issue = [&](int w) {  // one thread
    int m, bx, by, bz;
    decode(w, m, bx, by, bz);
    rhs_tma_issue<T, KB, 1>(buf, &bar[0], &a.map[m][0], &a.map[m][1], &a.map[m][2], bx, by, bz);
  };
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (tid == 0) issue(u0 + blockIdx.x);
  int it = 0;
  for (int w = u0 + blockIdx.x; w < u1; w += gridDim.x, ++it) {
    int m, bx, by, bz;
    decode(w, m, bx, by, bz);
    const BRhsRec<T>& b = a.r[m];
    const T forcing = (UPD == UPD_AB2) ? (T)(*b.forcing) : T(0);
    if (!rhs_tma_tile<T, FULL, UPD, KB, 1>(b.g, b.A[0], b.A[1], b.A[2], b.B[0], b.B[1], b.B[2], b.R[0], b.R[1],
                                           b.R[2], forcing, b.dt, UPD == UPD_FE ? 0 : b.have_hist, bx, by, bz, buf,
                                           &bar[0], (unsigned)it & 1u, pre, b.err, nullptr, 0u))
      return;
    __syncthreads();  // the stage and the constants are free for the next unit
    if (tid == 0 && w + (int)gridDim.x < u1) issue(w + gridDim.x);
  }
}

// CN of the members whose chunk count (nz over L-row chunks) is the same, one
// launch per chunk count: the block is (32, chunks) as in k_cn_solve, so no
// warp idles for a shallower member, one CTA per unit (component, column
// block), and what the tile reads of a member travels in the launch's
// __grid_constant__ parameter.  Every member's chunks are L rows (its
// tables' length), a compile-time constant as in k_cn_solve.
template <class T> struct BCnRec {
  T* B[3];  // u*, v*, w*, solved in place
  CnTab tab;
  const double* ubase;
  int nx, ny, nz, cgx;  // cgx: column blocks per component
};
template <class T> struct BatchCnArgs {
  BCnRec<T> r[TC_BATCH_MAX];
  int st[TC_BATCH_MAX + 1];  // first unit of each member of the class, then the end
  int n;
};
static_assert(sizeof(BatchCnArgs<double>) + 64 <= 32764, "kernel parameter limit");

template <class T, int L, int VEC> __device__ __forceinline__ void batch_cn_unit(const BatchCnArgs<T>& a) {
  const int w = blockIdx.x;
  if (w >= a.st[a.n]) return;
  const int m = batch_class_member(a.st, a.n, w);
  const BCnRec<T>& b = a.r[m];
  const int l = w - a.st[m];
  cn_tile<T, L, VEC, true>(b.B[0], b.B[1], b.B[2], b.tab, b.ubase, b.nx, b.ny, b.nz, l % b.cgx, l / b.cgx, L);
}
// FP32 storage, 16-row chunks: the packed sweeps under k_cn_solve_pk's bound
template <int MAXT>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT) kb_cn_pk(const __grid_constant__ BatchCnArgs<float> a) {
  batch_cn_unit<float, 16, 2>(a);
}
template <class T, int L, int MAXT>
__global__ void __launch_bounds__(MAXT) kb_cn_n(const __grid_constant__ BatchCnArgs<T> a) {
  batch_cn_unit<T, L, 1>(a);
}

// Register-FFT lengths of the ensemble kernels: N = 16 N1, N1 in {4, 6, 8, 12, 16}
// (64 .. 256 points), all with two rows per warp (128-thread x blocks).  The
// y transforms come in two sets, NMAX = 8 (every member's N1 <= 8) and
// NMAX = 16, since a kernel's registers are those of its longest transform;
// the x transforms take one launch per length.
__host__ __device__ constexpr bool batch_n1_ok(int n1) { return n1 == 4 || n1 == 6 || n1 == 8 || n1 == 12 || n1 == 16; }

template <int NMAX, class F> __device__ __forceinline__ void batch_n1_switch(int n1, F&& f) {
  if constexpr (NMAX <= 8) {
    switch (n1) {
      case 4: f(std::integral_constant<int, 4>{}); break;
      case 6: f(std::integral_constant<int, 6>{}); break;
      default: f(std::integral_constant<int, 8>{}); break;
    }
  } else {
    switch (n1) {
      case 4: f(std::integral_constant<int, 4>{}); break;
      case 6: f(std::integral_constant<int, 6>{}); break;
      case 8: f(std::integral_constant<int, 8>{}); break;
      case 12: f(std::integral_constant<int, 12>{}); break;
      default: f(std::integral_constant<int, 16>{}); break;
    }
  }
}

template <class T, int N1, bool INV>
__device__ __forceinline__ void batch_ffty_call(const BMember<T>* __restrict__ bp, int row0, cpx<double>* tiles) {
  const BMember<T>& b = *bp;
  ffty_rows<N1, INV>(b.X, b.nrows, b.twy, row0, tiles);
}

// The x transforms of the members whose nx is 16 N1, one launch per N1.
// What the transforms read of a member travels in the launch's
// __grid_constant__ parameter (uniform loads, no per-thread registers).
template <class T> struct BXRec {
  Grid<T> g;
  const T* B[3];  // u**, v**, w** (forward transform)
  cpx<double>* X;
  const cpx<double>* twx;
  double* p;
  double scale;
  int xgx;        // row blocks per plane
};
template <class T> struct BatchXArgs {
  BXRec<T> r[TC_BATCH_MAX];
  int st[TC_BATCH_MAX + 1];   // first inverse unit (row block, plane) of each member of the class, then the end
  int stf[TC_BATCH_MAX + 1];  // the same for the forward units (row block, group of TC_BATCH_XP planes)
  int n;
};
static_assert(sizeof(BatchXArgs<double>) + 64 <= 32764, "kernel parameter limit");

// Units are warp tasks of two rows; no block barrier.
template <class T, int NMAX, bool INV>
__global__ void __launch_bounds__(128, TC_BATCH_FFT_MINB) kb_ffty(const BMember<T>* __restrict__ M, int nm, int total, int tile_elems) {
  __shared__ int st[TC_BATCH_MAX + 1];
  batch_starts(M, nm, BK_FY, total, st);
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  cpx<double>* tiles = reinterpret_cast<cpx<double>*>(smraw) + (size_t)warp * 2 * tile_elems;
  for (int w = blockIdx.x * wpb + warp; w < total; w += gridDim.x * wpb) {
    const int m = batch_member(st, nm, w);
    const BMember<T>& b = M[m];
    const int row0 = (w - st[m]) * 2;
    batch_n1_switch<NMAX>(b.n1y, [&](auto I) { batch_ffty_call<T, decltype(I)::value, INV>(&b, row0, tiles); });
  }
}

// The z sweeps of every member's modes, one CTA of 64 threads per unit (as
// k_tri_lu2), what a sweep reads of its member in the launch's
// __grid_constant__ parameter: a persistent unit loop reading the member
// table from global memory spilled 428 bytes a thread at its register cap.
struct BTriRec {
  double* X;  // the spectrum, solved in place
  const double* rden;
  const double* cpt;
  PoissonTabs tb;
  int nxh, ny, nz;
};
struct BatchTriArgs {
  BTriRec r[TC_BATCH_MAX];
  int st[TC_BATCH_MAX + 1];  // first unit of each member, then the end
  int n;
};
__global__ void __launch_bounds__(64) kb_tri_n(const __grid_constant__ BatchTriArgs a) {
  const int w = blockIdx.x;
  if (w >= a.st[a.n]) return;
  const int m = batch_class_member(a.st, a.n, w);
  const BTriRec& b = a.r[m];
  tri_lu2_thread<8>(b.X, b.rden, b.cpt, b.tb, b.nxh, b.ny, b.nz, (w - a.st[m]) * 64 + threadIdx.x);
}

// Forward x transform of the members of one length N1: one CTA per unit of
// TC_BATCH_XP planes of a row block (units in the order of the plane groups,
// row blocks fastest).
template <class T, int N1>
__global__ void __launch_bounds__(128) kb_fftx_n(const __grid_constant__ BatchXArgs<T> a) {
  const int w = blockIdx.x;
  if (w >= a.stf[a.n]) return;
  const int m = batch_class_member(a.stf, a.n, w);
  const BXRec<T>& b = a.r[m];
  const int l = w - a.stf[m], bx = l % b.xgx, k0 = (l / b.xgx) * TC_BATCH_XP;
  const int k1 = min(k0 + TC_BATCH_XP, b.g.nz);
  for (int k = k0; k < k1; ++k) {
    if (k > k0) __syncthreads();  // the previous plane's spectra are read
    fftx_tile<T, N1, XROWS>(b.g, b.B[0], b.B[1], b.B[2], nullptr, b.X, b.twx, b.scale, bx, k);
  }
}

template <class T, int N1>
__global__ void __launch_bounds__(128) kb_ifftx_n(const __grid_constant__ BatchXArgs<T> a) {
  const int w = blockIdx.x;
  if (w >= a.st[a.n]) return;
  const int m = batch_class_member(a.st, a.n, w);
  const BXRec<T>& b = a.r[m];
  const int l = w - a.st[m];
  ifftx_tile<N1, XROWS>(b.X, b.p, b.g.ny, b.g.nz, b.twx, l % b.xgx, l / b.xgx);
}

// The projection of every member, one CTA per unit (a k_project_bulk
// block), what the tile reads of its member in the launch's
// __grid_constant__ parameter.  The member's last block (atomic ticket, per
// member) reduces its partials and updates its forcing, as in
// k_project_bulk.
template <class T> struct BProjRec {
  Grid<T> g;
  T* B[3];  // u**, v**, w**: corrected in place
  double* p;
  const double* dzf;
  BulkArgs ba;
  int pgx, pgy, pgz;  // block grid of k_project_bulk
};
template <class T> struct BatchProjArgs {
  BProjRec<T> r[TC_BATCH_MAX];
  int st[TC_BATCH_MAX + 1];  // first unit of each member, then the end
  int n;
};
static_assert(sizeof(BatchProjArgs<double>) + 64 <= 32764, "kernel parameter limit");

template <class T>
__global__ void __launch_bounds__(256) kb_proj_n(const __grid_constant__ BatchProjArgs<T> a) {
  const int w = blockIdx.x;
  if (w >= a.st[a.n]) return;
  const int m = batch_class_member(a.st, a.n, w);
  const BProjRec<T>& b = a.r[m];
  int l = w - a.st[m];
  const int bx = l % b.pgx;
  l /= b.pgx;
  const int by = l % b.pgy, bz = l / b.pgy;
  project_tile<T>(b.g, b.B[0], b.B[1], b.B[2], b.p, (double)b.ba.dt, b.dzf, b.ba, bx, by, bz, b.pgx, b.pgy, b.pgz);
}

}  // namespace tc
