// C ABI of the B200 TorChannel step (include/torchannel_b200.h): context,
// workspace carving, launch configuration and the extern "C" entry points.
// The library never allocates device memory; every buffer is carved from the
// caller's workspace.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/torchannel_b200.h"
#include "tc_common.cuh"
#include "tc_fft.cuh"
#include "tc_poisson.cuh"
#include "tc_poisson32.cuh"
#include "tc_stats.cuh"
#include "tc_step.cuh"
#include "tc_rhs_tma.cuh"
#include "tc_ffty_bulk.cuh"
#include "tc_adjoint.cuh"
#include "tc_batch.cuh"

using namespace tc;

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define TC_CUDA(call)                                                                     \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return fail(TC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TC_LAUNCHED()                                                                      \
  do {                                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                   \
    if (e_ != cudaSuccess) return fail(TC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------------------
// Workspace layout
// ---------------------------------------------------------------------------
struct Carver {
  size_t off = 0;
  char* base = nullptr;
  template <class P> P* take(size_t nbytes) {
    off = (off + 255) & ~(size_t)255;
    P* p = base ? reinterpret_cast<P*>(base + off) : nullptr;
    off += nbytes;
    return p;
  }
};

struct tc_ctx {
  int nx, ny, nz, nxh;
  int precision, top_neumann, rhs_fused;
  double Lx, Ly, Lz, nu, U_bulk, dx, dy;
  std::vector<double> dzf, dzc;
  int dev;
  size_t tsz;  // sizeof storage type
  // device buffers (storage type T unless noted)
  void* st[2][3];
  void* rh[3];
  double* p;             // pressure, FP64 in both precisions
  cpx<double>* X;        // spectral intermediate, FP64 in both precisions
  double* tri_rden; double* tri_cp;  // per-mode LU factors of the z systems
  double* tri_cpb;                    // c' below each chunk of k_yz_solve ([kx][16][ky])
  void* idzf_t; void* idzc_t;
  double* ubase_d; void* ubase_t;  // base profile of u (mixed precision)
  unsigned int* ticket;  // last-block counter of k_project_bulk
  double* dzf_d; double* dzc_d;
  double* k2x; double* k2y; double* cl; double* cr;
  cpx<double>* twx_d; cpx<double>* twy_d;
  CnTab tab;
  double* partials; double* partials2; int npart;
  double* scal;
  int* err;
  // statistics
  double* st_prof; double* st_spec; double* st_means; cpx<double>* st_S;
  int k_bot, k_top, stats_ready, n_samples;
  FftPlan planx, plany;
  int JT, RB, tri_bt, stats_RB, stats_CB;
  // fused y/z Poisson middle (k_yz_solve): cluster size, planes per CTA,
  // FFT batch rows, threads, shared memory; yz_ok = launchable here
  int yz_CS, yz_P, yz_FB, yz_thr, yz_ok, yz_on;
  int yzr_thr, yzr_ok;  // register-FFT form of the fused kernel (k_yz_solve_reg)
  // the Poisson middle as two streaming passes (k_ffty_fwd, k_bwd_iffty):
  // ys_ok = available for this grid, ys_on = used
  int ys_ok, ys_on;
  size_t yzr_smem;
  int nsm, yreg_blocks;  // SM count; resident-block cap of the y register FFT
  // y transforms with bulk-copy staging (k_ffty_bulk): available, used, grid
  int ybulk_ok, ybulk_on, ybulk_grid;
  int tri16_blocks;      // resident blocks of k_tri_lu2<16> on the device
  int cn_L_force;        // CN chunk length chosen by tc_set_cn_chunk (0: by nz)
  size_t yz_smem;
  int cur, have_hist, state_set;
  double tab_dt;
  // single-precision Poisson step (mixed contexts, tc_use_fp32_poisson): FP32
  // pressure pair (pf[pcur] = the last step's p, the base of the next solve;
  // the projection writes the new p into the other), FP32 factor tables and
  // y twiddles; the FP32 spectrum and the increment dp overlay X and p
  float* pf[2];
  float* rden32; float* cp32;
  cpx<float>* twy32;
  // RHS with tensor-copy staging (k_rhs_tma): maps of the u, v, w buffers of
  // both state parities, usable here, switched on, persistent CTAs
  CUtensorMap tmap[2][3];
  int rhs_tma_ok, rhs_tma_on, rhs_tma_grid, rhs_tma_mode;
  int pcur, p_hist, p_f32;  // pf[pcur] holds p; p of the last step is in pf (else in p)
  int psp_on, psp_ok, psp_warm, since_set;
  int yz32_thr;
  size_t yz32_smem;
  // adjoint: body force of the forward step (caller-owned, FP64 internal
  // layout, or null) and the dt of the CN adjoint tables in the scratch
  const double* body[3];
  double adj_tab_dt;
  const void* adj_tab_ptr;
  // per-step hooks of the adjoint driver (FP64): kinetic-energy accumulator
  // (weight read from device memory) and state tape (slot counter on device)
  double* ke_acc; const double* ke_w; double* ke_part;
  double* tape; int* tape_ctr; int tape_slots;
  // CUDA graph of two consecutive steps (tc_step replays it for n_steps >= 4)
  cudaStream_t cap_stream;
  cudaGraphExec_t gexec;
  int g_valid, g_scheme, g_cur, g_pcur, g_psp;
  double g_dt;
  int graphs_on;
  // per-phase timing ring (tc_timing_enable)
  int timing;
  int t_head, t_count;
  cudaEvent_t tev[TC_TIMING_RING][TC_NPHASE + 1];
  int tev_made;
};

// Record the boundary event `ph` of the current timed step.
static void mark(tc_ctx* c, int ph, cudaStream_t s) {
  if (c->timing) cudaEventRecord(c->tev[c->t_head][ph], s);
}

template <class T> static Grid<T> make_grid(const tc_ctx* c, int which_unused = 0) {
  (void)which_unused;
  Grid<T> g;
  g.nx = c->nx; g.ny = c->ny; g.nz = c->nz;
  g.idx = (T)(1.0 / c->dx); g.idy = (T)(1.0 / c->dy);
  g.nu_idx2 = (T)(c->nu * (1.0 / (c->dx * c->dx)));
  g.nu_idy2 = (T)(c->nu * (1.0 / (c->dy * c->dy)));
  g.nu = (T)c->nu;
  g.idzf = (const T*)c->idzf_t; g.idzc = (const T*)c->idzc_t;
  g.top_neumann = c->top_neumann; g.rhs_fused = c->rhs_fused;
  const bool mixed = c->precision == TC_MIXED;
  g.ubase_t = mixed ? (const T*)c->ubase_t : nullptr;
  g.ubase_d = mixed ? c->ubase_d : nullptr;
  return g;
}

static size_t carve(tc_ctx* c, char* base) {
  Carver cv; cv.base = base;
  const size_t n = (size_t)c->nx * c->ny;
  const size_t ncell = n * c->nz, nface = n * (c->nz + 1);
  const size_t T_ = c->tsz;
  for (int s = 0; s < 2; ++s) {
    c->st[s][0] = cv.take<char>(ncell * T_);
    c->st[s][1] = cv.take<char>(ncell * T_);
    c->st[s][2] = cv.take<char>(nface * T_);
  }
  c->rh[0] = cv.take<char>(ncell * T_);
  c->rh[1] = cv.take<char>(ncell * T_);
  c->rh[2] = cv.take<char>(nface * T_);
  c->p = cv.take<double>(ncell * 8);
  const size_t nspec = (size_t)c->nxh * c->nz * c->ny;
  c->X = cv.take<cpx<double>>(nspec * 16);
  c->tri_rden = cv.take<double>(nspec * 8);
  c->tri_cp = cv.take<double>(nspec * 8);
  c->tri_cpb = cv.take<double>((size_t)c->nxh * 16 * c->ny * 8);
  c->idzf_t = cv.take<char>(c->nz * T_);
  c->idzc_t = cv.take<char>((c->nz + 1) * T_);
  c->ubase_d = cv.take<double>(c->nz * 8);
  c->ubase_t = cv.take<char>(c->nz * T_);
  c->ticket = cv.take<unsigned int>(256);
  c->dzf_d = cv.take<double>(c->nz * 8);
  c->dzc_d = cv.take<double>((c->nz + 1) * 8);
  c->k2x = cv.take<double>(c->nxh * 8);
  c->k2y = cv.take<double>(c->ny * 8);
  c->cl = cv.take<double>(c->nz * 8);
  c->cr = cv.take<double>(c->nz * 8);
  c->twx_d = cv.take<cpx<double>>(c->nx * 16);
  c->twy_d = cv.take<cpx<double>>(c->ny * 16);
  c->tab.uv = cv.take<double>(8 * c->nz * 8);
  c->tab.w = cv.take<double>(8 * c->nz * 8);
  c->tab.beta = cv.take<double>(8);
  c->tab.corr = cv.take<double>(c->nz * 8);
  const int gx = (c->nx + 31) / 32, gy = (c->ny + 7) / 8;
  c->npart = gx * gy * (c->nz + 1);
  c->partials = cv.take<double>((size_t)c->npart * 8);
  c->partials2 = cv.take<double>((size_t)c->npart * 8);
  c->scal = cv.take<double>(SC_COUNT * 8);
  c->err = cv.take<int>(64);
  c->st_prof = cv.take<double>(5 * c->nz * 8);
  c->st_spec = cv.take<double>((size_t)4 * (c->nx / 2) * (c->ny / 2) * 8);
  c->st_means = cv.take<double>(3 * c->nz * 8);
  c->st_S = cv.take<cpx<double>>(3 * n * 16);
  if (c->precision == TC_MIXED) {
    c->pf[0] = cv.take<float>(ncell * 4);
    c->pf[1] = cv.take<float>(ncell * 4);
    c->rden32 = cv.take<float>(nspec * 4);
    c->cp32 = cv.take<float>(nspec * 4);
    c->twy32 = cv.take<cpx<float>>((size_t)c->ny * 8);
  }
  return cv.off + 256;
}

static int validate(const tc_grid_desc* g) {
  if (!g) return fail(TC_ERR_ARG, "null grid descriptor");
  if (g->nx < 8 || g->ny < 8 || g->nz < 4) return fail(TC_ERR_SIZE, "nx, ny must be >= 8 and nz >= 4");
  if ((g->nx & 1) || (g->ny & 1)) return fail(TC_ERR_SIZE, "nx and ny must be even");
  if (g->nz > 512) return fail(TC_ERR_SIZE, "nz must be <= 512");
  FftPlan a, b;
  if (!fft_make_plan(g->nx, &a) || !fft_make_plan(g->ny, &b))
    return fail(TC_ERR_SIZE, "nx and ny must factor into 2 and 3 only");
  if (g->nx > 4096 || g->ny > 4096) return fail(TC_ERR_SIZE, "nx, ny must be <= 4096");
  // kernels index within a field in 32 bits; such a grid (> 200 GB of state)
  // does not fit on one device in any case
  if ((uint64_t)g->nx * g->ny * (g->nz + 1) >= (1ull << 32))
    return fail(TC_ERR_SIZE, "nx * ny * (nz + 1) must be below 2^32");
  if (g->precision != TC_FP64 && g->precision != TC_MIXED) return fail(TC_ERR_ARG, "bad precision");
  if (!g->dz_f || !g->dz_c) return fail(TC_ERR_ARG, "null dz_f / dz_c");
  if (!(g->Lx > 0 && g->Ly > 0 && g->Lz > 0 && g->nu > 0)) return fail(TC_ERR_ARG, "non-positive domain or viscosity");
  return TC_OK;
}

static void fill_basic(tc_ctx* c, const tc_grid_desc* g) {
  c->nx = g->nx; c->ny = g->ny; c->nz = g->nz; c->nxh = g->nx / 2 + 1;
  c->precision = g->precision; c->top_neumann = g->top_wall == TC_TOP_FREESLIP;
  c->rhs_fused = g->rhs_path == TC_RHS_FUSED;
  c->Lx = g->Lx; c->Ly = g->Ly; c->Lz = g->Lz; c->nu = g->nu; c->U_bulk = g->U_bulk;
  c->dx = g->Lx / g->nx; c->dy = g->Ly / g->ny;
  c->tsz = g->precision == TC_FP64 ? 8 : 4;
  fft_make_plan(g->nx, &c->planx);
  fft_make_plan(g->ny, &c->plany);
  // launch shapes: x transform rows per block (even divisor of ny, smem <= 100 KB)
  int JT = 16;
  while (JT > 2 && (c->ny % JT != 0 || ((size_t)2 * (JT / 2) * padded_len<double>(c->nx) + c->nx) * 16 > 100 * 1024))
    JT -= 2;
  c->JT = JT;
  int RB = 8;
  while (RB > 1 && ((size_t)2 * RB * padded_len<double>(c->ny) + c->ny) * 16 > 100 * 1024) RB /= 2;
  c->RB = RB;
  c->tri_bt = (64 * (size_t)c->nz * 8 <= 200 * 1024) ? 64 : 32;
  int sRB = 8;
  while (sRB > 1 && ((size_t)2 * sRB * padded_len<double>(c->nx) + c->nx) * 16 > 100 * 1024) sRB /= 2;
  c->stats_RB = sRB;
  int sCB = 8;
  while (sCB > 1 && ((size_t)2 * sCB * padded_len<double>(c->ny) + c->ny) * 16 > 100 * 1024) sCB /= 2;
  c->stats_CB = sCB;
  // fused y/z middle: clusters of CS CTAs (power of two, <= 16) of about 16
  // planes each, the FFT scratch shrunk until a CTA fits in 200 KB
  int CS = 1;
  while (CS < 16 && CS * 16 < c->nz) CS *= 2;
  const int P = (c->nz + CS - 1) / CS;
  int FB = P < 8 ? P : 8;
  auto yz_bytes = [&](int fb) {
    return (size_t)(P + fb) * padded_len<double>(c->ny) * 16 + (size_t)c->ny * 16 + (size_t)6 * c->ny * 8;
  };
  while (FB > 1 && yz_bytes(FB) > 200 * 1024) FB /= 2;
  c->yz_CS = CS; c->yz_P = P; c->yz_FB = FB;
  c->yz_thr = ((c->ny + 31) / 32) * 32;  // one thread per column ky
  if (c->yz_thr < 256) c->yz_thr = 256;
  c->yz_smem = yz_bytes(FB);
  c->yz_ok = 0; c->yz_on = 0;
  c->ys_ok = 0; c->ys_on = 0;
  c->ybulk_ok = 0; c->ybulk_on = 0; c->ybulk_grid = 1;
}

extern "C" const char* tc_version(void) { return "torchannel_b200 0.1 (sm_100a)"; }
extern "C" const char* tc_last_error(void) { return g_err.c_str(); }

extern "C" int tc_workspace_bytes(const tc_grid_desc* g, size_t* bytes) {
  int rc = validate(g);
  if (rc) return rc;
  if (!bytes) return fail(TC_ERR_ARG, "null bytes");
  tc_ctx c{};
  fill_basic(&c, g);
  *bytes = carve(&c, nullptr);
  return TC_OK;
}

// ---- register-FFT launches (lengths 16 K, K as rowfft_supported) ----
template <class F> static void for_each_n1(int n, F&& f) {
  switch (n / 16) {
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 12: f(std::integral_constant<int, 12>{}); break;
    case 9: f(std::integral_constant<int, 9>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    case 18: f(std::integral_constant<int, 18>{}); break;
    case 24: f(std::integral_constant<int, 24>{}); break;
    case 32: f(std::integral_constant<int, 32>{}); break;
    case 36: f(std::integral_constant<int, 36>{}); break;
    case 48: f(std::integral_constant<int, 48>{}); break;
    default: f(std::integral_constant<int, 64>{}); break;
  }
}
template <int N1> static size_t fftx_reg_smem() {
  return (size_t)(XROWS / 2) * ((RowFft<N1>::TILE + 7) / 8 * 8 + 1) * sizeof(cpx<double>);
}
template <int N1> static size_t ifftx_reg_smem() {
  return (size_t)XROWS * ifftx_pitch<N1>() * sizeof(cpx<double>);
}
template <int N1> static int xreg_threads() { return 16 * XROWS / RowFft<N1>::RPW; }
template <int N1> static size_t ffty_reg_smem() {
  return (size_t)4 * RowFft<N1>::RPW * RowFft<N1>::TILE * sizeof(cpx<double>);
}
// x transforms take the register path for supported nx when ny is a multiple
// of 16 (16 rows a block); y transforms for supported ny.
static bool xreg_ok(const tc_ctx* c) { return rowfft_supported(c->nx) && c->ny % XROWS == 0; }
static bool yreg_ok(const tc_ctx* c) { return rowfft_supported(c->ny); }

// The streamed y / z passes (k_ffty_fwd, k_bwd_iffty): register y transforms
// of at most 256 points (one sweep column per thread).
static bool ys_supported(const tc_ctx* c) { return yreg_ok(c) && c->ny <= 256; }

// Shared-memory opt-in and the resident-block count of the y kernel.
template <class T> static int reg_fft_setup(tc_ctx* c) {
  int rc = TC_OK;
  if (xreg_ok(c)) {
    for_each_n1(c->nx, [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      if (cudaFuncSetAttribute(k_div_fftx_reg<T, N1, XROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)fftx_reg_smem<N1>()) != cudaSuccess ||
          cudaFuncSetAttribute(k_ifftx_reg<N1, XROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ifftx_reg_smem<N1>()) != cudaSuccess)
        rc = fail(TC_ERR_CUDA, "register x FFT attributes");
    });
  }
  c->yreg_blocks = c->nsm;
  if (yreg_ok(c)) {
    for_each_n1(c->ny, [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      int nb = 0;
      if (cudaFuncSetAttribute(k_ffty_reg<N1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ffty_reg_smem<N1>()) != cudaSuccess ||
          cudaFuncSetAttribute(k_ffty_reg<N1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ffty_reg_smem<N1>()) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ffty_reg<N1, false>, 128, ffty_reg_smem<N1>()) !=
              cudaSuccess)
        rc = fail(TC_ERR_CUDA, "register y FFT setup");
      if (nb > 0) c->yreg_blocks = nb * c->nsm;
    });
  }
  if (c->yreg_blocks < 1) c->yreg_blocks = 1;
  c->ybulk_ok = 0;
  if (yreg_ok(c)) {
    for_each_n1(c->ny, [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      const int sm = (int)YBulk<N1>::smem();
      int nb = 0;
      if (cudaFuncSetAttribute(k_ffty_bulk<N1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
              cudaSuccess &&
          cudaFuncSetAttribute(k_ffty_bulk<N1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
              cudaSuccess &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ffty_bulk<N1, false>, 128, sm) == cudaSuccess &&
          nb >= 1) {
        c->ybulk_ok = 1;
        c->ybulk_grid = nb * c->nsm;
      }
    });
    cudaGetLastError();
  }
  {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_tri_lu2<16>, 64, 0) != cudaSuccess)
      rc = fail(TC_ERR_CUDA, "z solve occupancy");
    c->tri16_blocks = nb * c->nsm;
  }
  c->ys_ok = 0;
  if (ys_supported(c)) {
    for_each_n1(c->ny, [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      if constexpr (YzPass<N1>::CPT == 1) {
        const int sm = (int)YzPass<N1>::smem();
        if (cudaFuncSetAttribute(k_ffty_fwd<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess ||
            cudaFuncSetAttribute(k_bwd_iffty<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess)
          rc = fail(TC_ERR_CUDA, "streamed y / z pass attributes");
        else
          c->ys_ok = 1;
      }
    });
  }
  return rc;
}


template <bool BWD> static void ys_pass(const tc_ctx* c, cpx<double>* X, cudaStream_t s) {
  for_each_n1(c->ny, [&](auto I) {
    constexpr int N1 = decltype(I)::value;
    if constexpr (YzPass<N1>::CPT == 1) {
      if (BWD)
        k_bwd_iffty<N1><<<c->nxh, YzPass<N1>::NT, YzPass<N1>::smem(), s>>>(X, c->tri_cp, c->twy_d, c->nz);
      else
        k_ffty_fwd<N1><<<c->nxh, YzPass<N1>::NT, YzPass<N1>::smem(), s>>>(X, c->tri_rden, c->cl, c->twy_d, c->nz);
    }
  });
}

template <bool INV> static void ffty_reg(const tc_ctx* c, cpx<double>* X, int nrows, cudaStream_t s) {
  for_each_n1(c->ny, [&](auto I) {
    constexpr int N1 = decltype(I)::value;
    if (c->ybulk_on) {
      const int ntiles = (nrows + YBulk<N1>::R - 1) / YBulk<N1>::R;
      k_ffty_bulk<N1, INV><<<std::min(ntiles, c->ybulk_grid), 128, YBulk<N1>::smem(), s>>>(X, nrows, c->twy_d,
                                                                                          c->err);
      return;
    }
    const int rpb = 4 * RowFft<N1>::RPW;
    int nblk = (nrows + rpb - 1) / rpb;
    if (nblk > c->yreg_blocks) nblk = c->yreg_blocks;
    k_ffty_reg<N1, INV><<<nblk, 128, ffty_reg_smem<N1>(), s>>>(X, nrows, c->twy_d);
  });
}

template <class T>
static void fftx_reg(const tc_ctx* c, Grid<T> g, const T* u, const T* v, const T* w, const double* field,
                     cpx<double>* X, double scale, cudaStream_t s) {
  for_each_n1(c->nx, [&](auto I) {
    constexpr int N1 = decltype(I)::value;
    k_div_fftx_reg<T, N1, XROWS><<<dim3(c->ny / XROWS, c->nz), xreg_threads<N1>(), fftx_reg_smem<N1>(), s>>>(
        g, u, v, w, field, X, c->twx_d, scale);
  });
}

static void ifftx_reg(const tc_ctx* c, const cpx<double>* X, double* p, cudaStream_t s) {
  for_each_n1(c->nx, [&](auto I) {
    constexpr int N1 = decltype(I)::value;
    k_ifftx_reg<N1, XROWS><<<dim3(c->ny / XROWS, c->nz), xreg_threads<N1>(), ifftx_reg_smem<N1>(), s>>>(
        X, p, c->ny, c->nz, c->twx_d);
  });
}

// Fused y/z middle with register transforms: threads (one per column ky, at
// least 8 warps) and shared memory (rows, per-warp transpose tiles, chunk ends).
template <int N1> static size_t yzr_bytes(int P, int thr) {
  using RF = RowFft<N1>;
  return ((size_t)P * RF::N + (size_t)(thr / 32) * RF::RPW * RF::TILE + 2 * (size_t)RF::N) * sizeof(cpx<double>) +
         2 * (size_t)RF::N * sizeof(double);
}
template <int N1, int PM> static void* yzr_kernel() { return (void*)k_yz_solve_reg<N1, PM>; }
static void* yzr_fn(const tc_ctx* c) {
  void* f = nullptr;
  for_each_n1(c->ny, [&](auto I) {
    constexpr int N1 = decltype(I)::value;
    f = c->yz_P <= 16 ? yzr_kernel<N1, 16>() : yzr_kernel<N1, 32>();
  });
  return f;
}

static cudaLaunchConfig_t yz_config(const tc_ctx* c, cudaLaunchAttribute* at, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(c->nxh * c->yz_CS, 1, 1);
  cfg.blockDim = dim3(c->yz_thr, 1, 1);
  cfg.dynamicSmemBytes = c->yz_smem;
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = c->yz_CS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

// Whether the cluster shape of k_yz_solve_reg can be resident on this device
// (sets its attributes first).
static int yzr_probe(tc_ctx* c) {
  if (!rowfft_supported(c->ny) || c->yz_P > 32) return 0;
  c->yzr_thr = ((c->ny + 31) / 32) * 32;
  if (c->yzr_thr < 256) c->yzr_thr = 256;
  for_each_n1(c->ny, [&](auto I) {
    constexpr int N1 = decltype(I)::value;
    c->yzr_smem = yzr_bytes<N1>(c->yz_P, c->yzr_thr);
  });
  if (c->yzr_thr > 512 || c->yzr_smem > 200 * 1024) return 0;
  void* f = yzr_fn(c);
  if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
      cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = yz_config(c, at, 0);
  cfg.blockDim = dim3(c->yzr_thr, 1, 1);
  cfg.dynamicSmemBytes = c->yzr_smem;
  int ncl = 0;
  if (cudaOccupancyMaxActiveClusters(&ncl, f, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return ncl > 0;
}

// Whether the cluster shape of k_yz_solve can be resident on this device.
static int yz_probe(tc_ctx* c) {
  if (c->yz_smem > 200 * 1024 || c->yz_thr > 512 || c->yz_P > 32) return 0;
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = yz_config(c, at, 0);
  int ncl = 0;
  cudaError_t e = c->yz_P <= 16 ? cudaOccupancyMaxActiveClusters(&ncl, k_yz_solve<16>, &cfg)
                                : cudaOccupancyMaxActiveClusters(&ncl, k_yz_solve<32>, &cfg);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return ncl > 0;
}

// The CN kernel of 16-row chunks: the packed FP32 sweeps (two columns a
// thread) for FP32 storage, one FP64 column a thread otherwise.
template <class T, bool FIXED> static auto cn16_kernel() {
  if constexpr (sizeof(T) == 4)
    return k_cn_solve_pk<16, 512, FIXED>;
  else
    return k_cn_solve<double, 16, 1, 512, FIXED>;
}

template <class T> static int set_smem_attrs(const tc_ctx* c) {
  const int big = 200 * 1024;
  TC_CUDA(cudaFuncSetAttribute(k_div_fftx<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_ifftx, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_ffty<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_ffty<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_tri, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_yz_solve<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_yz_solve<16>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  TC_CUDA(cudaFuncSetAttribute(k_yz_solve<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_yz_solve<32>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  TC_CUDA(cudaFuncSetAttribute(cn16_kernel<T, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(cn16_kernel<T, false>(), cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_cn_solve<T, 32, 1, 512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_cn_solve<T, 32, 1, 512, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_fft_cols<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TC_CUDA(cudaFuncSetAttribute(k_fft_rows_d<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  (void)c;
  return TC_OK;
}

// ---- single-precision Poisson step (mixed contexts) ----------------------
// k_yz32 lengths: ny = 16 K with a register transform and K <= 24 (N <= 384).
template <class F> static void for_each_yz32(int n, F&& f) {
  switch (n / 16) {
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 9: f(std::integral_constant<int, 9>{}); break;
    case 12: f(std::integral_constant<int, 12>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    case 18: f(std::integral_constant<int, 18>{}); break;
    case 24: f(std::integral_constant<int, 24>{}); break;
    default: break;
  }
}
static bool yz32_len_ok(int ny) { return rowfft_supported(ny) && ny / 16 <= 24; }
static bool psp_ready(const tc_ctx* c) { return c->psp_on && c->p_hist >= 1 && c->since_set >= c->psp_warm; }

template <class T> static void to_t(const std::vector<double>& src, std::vector<unsigned char>& dst) {
  dst.resize(src.size() * sizeof(T));
  T* d = reinterpret_cast<T*>(dst.data());
  for (size_t e = 0; e < src.size(); ++e) d[e] = (T)src[e];
}

static int upload(void* dptr, const std::vector<double>& v, size_t tsz) {
  if (tsz == 8) {
    TC_CUDA(cudaMemcpy(dptr, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
  } else {
    std::vector<unsigned char> b;
    to_t<float>(v, b);
    TC_CUDA(cudaMemcpy(dptr, b.data(), b.size(), cudaMemcpyHostToDevice));
  }
  return TC_OK;
}

static std::vector<double> twiddles(int n) {
  std::vector<double> t(2 * (size_t)n);
  const double pi = 3.14159265358979323846264338327950288;
  for (int m = 0; m < n; ++m) {
    // exp(-2 pi i m / n); use symmetric reduction for accuracy
    double ang = -2.0 * pi * (double)m / (double)n;
    t[2 * m] = std::cos(ang);
    t[2 * m + 1] = std::sin(ang);
  }
  return t;
}

// ---- RHS with tensor-copy staging ----------------------------------------
typedef CUresult (*TensorMapEncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                           const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                           CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                           CUtensorMapFloatOOBfill);

// Shapes of the tensor-copy RHS: planes per tile, stages, resident CTAs per
// SM the registers are bounded for.
template <class T, int KB, int NST, int MINB> struct RhsV {
  using S = RhsTma<T, KB, NST>;
  static constexpr int kb = KB, nst = NST;
  template <bool FULL, int UPD> static constexpr auto fn() { return k_rhs_tma<T, FULL, UPD, KB, NST, MINB>; }
};
// Shapes (planes per tile, stages, resident CTAs per SM) by mode, FP32 /
// FP64 storage: 1: 8, 1, 3 / 2, 1, 5 (the default); 2: 4, 1, 4 / 2, 1, 4;
// 3: 8, 1, 4 / 4, 1, 3; 4: 16, 1, 2 / 4, 2, 2 (the persistent two-stage
// pipeline); 5: 8, 2, 2 and 6: 4, 2, 4 (FP32 only; two-stage pipelines).
// Measured at 192 x 192 x 128 (us of the kernel, FP32 column march / FP64
// per-plane stencils): mode 1 63.5 / 111.3 (64.7 before the march's per-tile
// constants were staged in shared memory), mode 2 66.8, mode 3 70.0 (64
// registers, spills), mode 4 67.9 / 121.5, mode 5 70.5 (108 registers),
// mode 6 71.4; per-thread staging (k_rhs_update) 91.5 / 117.7.
template <class T, class F> static void rhs_variant(int mode, F&& f) {
  if constexpr (sizeof(T) == 8) {
    switch (mode) {
      case 2: f(RhsV<double, 2, 1, 4>{}); break;
      case 3: f(RhsV<double, 4, 1, 3>{}); break;
      case 4: f(RhsV<double, 4, 2, 2>{}); break;
      default: f(RhsV<double, 2, 1, 5>{}); break;
    }
  } else {
    switch (mode) {
      case 2: f(RhsV<float, 4, 1, 4>{}); break;
      case 3: f(RhsV<float, 8, 1, 4>{}); break;
      case 4: f(RhsV<float, 16, 1, 2>{}); break;
      case 5: f(RhsV<float, 8, 2, 2>{}); break;
      case 6: f(RhsV<float, 4, 2, 4>{}); break;
      default: f(RhsV<float, 8, 1, 3>{}); break;
    }
  }
}

// Tensor maps of the six state buffers (3-D: x, y, planes; boxes of the
// k_rhs_tma tile of shape `mode`), kernel attributes and the grid.  Leaves
// rhs_tma_ok = 0 (the staged kernel k_rhs_update runs) where the grid does
// not allow it: x rows must be a multiple of 16 bytes and the domain at least
// two tiles wide.
template <class T> static int rhs_tma_setup(tc_ctx* c, int mode) {
  c->rhs_tma_ok = 0;
  c->rhs_tma_on = 0;
  if (((size_t)c->nx * sizeof(T)) % 16 != 0 || c->nx < 2 * RHS_TX || c->ny < 16) return TC_OK;
  static TensorMapEncodeTiledFn enc = nullptr;
  if (!enc) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f) {
      cudaGetLastError();
      return TC_OK;
    }
    enc = (TensorMapEncodeTiledFn)f;
  }
  bool ok = true;
  rhs_variant<T>(mode, [&](auto V) {
    using VV = decltype(V);
    using S = typename VV::S;
    const CUtensorMapDataType dty = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    for (int st = 0; st < 2 && ok; ++st)
      for (int f = 0; f < 3 && ok; ++f) {
        const cuuint64_t gdim[3] = {(cuuint64_t)c->nx, (cuuint64_t)c->ny,
                                    (cuuint64_t)(f == 2 ? c->nz + 1 : c->nz)};
        const cuuint64_t gstr[2] = {(cuuint64_t)c->nx * sizeof(T), (cuuint64_t)c->nx * c->ny * sizeof(T)};
        const cuuint32_t box[3] = {(cuuint32_t)S::BX, (cuuint32_t)S::BY, (cuuint32_t)S::BZ};
        const cuuint32_t est[3] = {1, 1, 1};
        ok = enc(&c->tmap[st][f], dty, 3, c->st[st][f], gdim, gstr, box, est, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
      }
    const int sm = (int)S::smem();
    int nb = 0;
    ok = ok &&
         cudaFuncSetAttribute(VV::template fn<false, UPD_AB2>(), cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
             cudaSuccess &&
         cudaFuncSetAttribute(VV::template fn<true, UPD_AB2>(), cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
             cudaSuccess &&
         cudaFuncSetAttribute(VV::template fn<true, UPD_FE>(), cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
             cudaSuccess &&
         cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, VV::template fn<false, UPD_AB2>(), RHS_TX * S::TY, sm) ==
             cudaSuccess &&
         nb >= 1;
    if (!ok) return;
    int ntx, nty, ntz;
    rhs_tma_tiles(c->nx, c->ny, c->nz, VV::kb, &ntx, &nty, &ntz);
    c->rhs_tma_grid = VV::nst == 2 ? std::min(ntx * nty * ntz, nb * c->nsm) : ntx * nty * ntz;
  });
  if (!ok) {
    cudaGetLastError();
    return TC_OK;
  }
  c->rhs_tma_mode = mode;
  c->rhs_tma_ok = 1;
  c->rhs_tma_on = 1;
  return TC_OK;
}

template <class T, bool FULL, int UPD>
static void launch_rhs_tma(const tc_ctx* c, const Grid<T>& g, T* const* A, T* const* B, T* const* R, double dt,
                           int have_hist, cudaStream_t s) {
  rhs_variant<T>(c->rhs_tma_mode, [&](auto V) {
    using VV = decltype(V);
    using S = typename VV::S;
    int ntx, nty, ntz;
    rhs_tma_tiles(c->nx, c->ny, c->nz, VV::kb, &ntx, &nty, &ntz);
    const CUtensorMap* m = c->tmap[c->cur];
    VV::template fn<FULL, UPD>()<<<c->rhs_tma_grid, dim3(RHS_TX, S::TY), S::smem(), s>>>(
        m[0], m[1], m[2], g, A[0], A[1], A[2], B[0], B[1], B[2], R[0], R[1], R[2], c->scal + SC_FORCING, (T)dt,
        have_hist, ntx, nty, ntz, c->err);
  });
}

// Whether the single-precision Poisson step can run on this grid (register x
// transforms, a k_yz32 length, the kx slab within a CTA's shared memory),
// and its tables and kernel attributes.
static int psp_setup(tc_ctx* c, const std::vector<double>& twy) {
  c->psp_ok = 0; c->psp_on = 0; c->psp_warm = 10;
  if (c->precision != TC_MIXED || !xreg_ok(c) || !yz32_len_ok(c->ny)) return TC_OK;
  int optin = 0;
  TC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
  c->yz32_smem = yz32_smem_bytes(c->ny, c->nz);
  if (c->yz32_smem > (size_t)optin) return TC_OK;
  int rc = TC_OK;
  for_each_yz32(c->ny, [&](auto I) {
    constexpr int K = decltype(I)::value;
    c->yz32_thr = yz32_threads<K>();
    if (cudaFuncSetAttribute(k_yz32<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->yz32_smem) !=
        cudaSuccess)
      rc = fail(TC_ERR_CUDA, "k_yz32 attributes");
  });
  if (rc) return rc;
  for_each_n1(c->nx, [&](auto I) {
    constexpr int N1 = decltype(I)::value;
    if (cudaFuncSetAttribute(k_div_fftx_reg32<float, N1, XROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fftx_reg_smem<N1>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_ifftx_reg32<N1, XROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ifftx_reg_smem<N1>()) != cudaSuccess)
      rc = fail(TC_ERR_CUDA, "single-precision x transform attributes");
  });
  if (rc) return rc;
  const size_t nspec = (size_t)c->nxh * c->nz * c->ny;
  k_tri_factors32<<<(unsigned)((nspec + 255) / 256 < 4096 ? (nspec + 255) / 256 : 4096), 256>>>(
      c->tri_rden, c->tri_cp, c->rden32, c->cp32, nspec);
  if (cudaGetLastError() != cudaSuccess) return fail(TC_ERR_CUDA, "FP32 factor tables launch");
  if ((rc = upload(c->twy32, twy, 4))) return rc;
  c->psp_ok = 1;
  return TC_OK;
}

extern "C" int tc_create(const tc_grid_desc* g, void* workspace, size_t bytes, tc_ctx** out) {
  int rc = validate(g);
  if (rc) return rc;
  if (!out || !workspace) return fail(TC_ERR_ARG, "null workspace / out");
  if (((uintptr_t)workspace) & 255) return fail(TC_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  tc_ctx* c = new tc_ctx();
  fill_basic(c, g);
  size_t need = carve(c, (char*)workspace);
  if (bytes < need) { delete c; return fail(TC_ERR_WORKSPACE, "workspace too small"); }
  cudaGetDevice(&c->dev);
  c->dzf.assign(g->dz_f, g->dz_f + g->nz);
  c->dzc.assign(g->dz_c, g->dz_c + g->nz + 1);
  auto bail = [&](int r) { delete c; return r; };
  if (cudaMemset(workspace, 0, need) != cudaSuccess) return bail(fail(TC_ERR_CUDA, "memset workspace"));
  std::vector<double> idzf(c->nz), idzc(c->nz + 1), cl(c->nz), cr(c->nz);
  for (int k = 0; k < c->nz; ++k) idzf[k] = 1.0 / c->dzf[k];
  for (int k = 0; k <= c->nz; ++k) idzc[k] = 1.0 / c->dzc[k];
  for (int k = 0; k < c->nz; ++k) {
    cl[k] = 1.0 / (c->dzc[k] * c->dzf[k]);
    cr[k] = 1.0 / (c->dzc[k + 1] * c->dzf[k]);
  }
  // modified wavenumbers (projection_fft.py:26-39): kx = 2 pi m / (nx dx), k~ = (2/dx) sin(kx dx / 2)
  const double pi = 3.14159265358979323846264338327950288;
  std::vector<double> k2x(c->nxh), k2y(c->ny);
  for (int m = 0; m < c->nxh; ++m) {
    double f = (m < (c->nx + 1) / 2 ? (double)m : (double)(m - c->nx)) / ((double)c->nx * (c->dx / (2 * pi)));
    double km = (2.0 / c->dx) * std::sin(f * c->dx / 2.0);
    k2x[m] = km * km;
  }
  for (int m = 0; m < c->ny; ++m) {
    double f = (m < (c->ny + 1) / 2 ? (double)m : (double)(m - c->ny)) / ((double)c->ny * (c->dy / (2 * pi)));
    double km = (2.0 / c->dy) * std::sin(f * c->dy / 2.0);
    k2y[m] = km * km;
  }
  std::vector<double> twx = twiddles(c->nx), twy = twiddles(c->ny);
  int r2 = TC_OK;
  if ((r2 = upload(c->idzf_t, idzf, c->tsz)) || (r2 = upload(c->idzc_t, idzc, c->tsz)) ||
      (r2 = upload(c->dzf_d, c->dzf, 8)) || (r2 = upload(c->dzc_d, c->dzc, 8)) ||
      (r2 = upload(c->k2x, k2x, 8)) || (r2 = upload(c->k2y, k2y, 8)) || (r2 = upload(c->cl, cl, 8)) ||
      (r2 = upload(c->cr, cr, 8)) || (r2 = upload(c->twx_d, twx, 8)) || (r2 = upload(c->twy_d, twy, 8)))
    return bail(r2);
  r2 = (c->tsz == 8) ? set_smem_attrs<double>(c) : set_smem_attrs<float>(c);
  if (r2) return bail(r2);
  if (cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev) != cudaSuccess)
    return bail(fail(TC_ERR_CUDA, "SM count"));
  r2 = (c->tsz == 8) ? reg_fft_setup<double>(c) : reg_fft_setup<float>(c);
  if (r2) return bail(r2);
  {
    PoissonTabs tb{c->k2x, c->k2y, c->cl, c->cr};
    const int nmodes = c->nxh * c->ny;
    k_tri_factors<<<(nmodes + 127) / 128, 128>>>(tb, c->tri_rden, c->tri_cp, c->nxh, c->ny, c->nz);
    if (cudaGetLastError() != cudaSuccess) return bail(fail(TC_ERR_CUDA, "tri factors launch"));
  }
  if ((r2 = psp_setup(c, twy))) return bail(r2);
  r2 = (c->tsz == 8) ? rhs_tma_setup<double>(c, 1) : rhs_tma_setup<float>(c, 1);
  if (r2) return bail(r2);
  c->yz_ok = yz_probe(c);
  c->yzr_ok = c->yz_ok ? yzr_probe(c) : 0;
  c->yz_on = 0;  // the three-kernel path with register FFTs is faster
  c->ys_on = 0;  // so far also than the two streaming passes
  c->ybulk_on = 0;  // measured slower than the per-lane loads with register prefetch
  if (c->yz_ok) {
    PoissonTabs tb{c->k2x, c->k2y, c->cl, c->cr};
    const int nmodes = c->nxh * c->ny;
    k_tri_chunk_cp<<<(nmodes + 127) / 128, 128>>>(tb, c->tri_cpb, c->nxh, c->ny, c->nz, c->yz_CS, c->yz_P);
    if (cudaGetLastError() != cudaSuccess) return bail(fail(TC_ERR_CUDA, "chunk factors launch"));
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(TC_ERR_CUDA, "create sync"));
  c->tab_dt = -1.0;
  c->adj_tab_dt = -1.0;
  c->adj_tab_ptr = nullptr;
  c->ke_acc = nullptr; c->ke_w = nullptr; c->ke_part = nullptr;
  c->tape = nullptr; c->tape_ctr = nullptr; c->tape_slots = 0;
  c->body[0] = c->body[1] = c->body[2] = nullptr;
  c->graphs_on = 1;
  *out = c;
  return TC_OK;
}

extern "C" int tc_destroy(tc_ctx* ctx) {
  if (ctx && ctx->g_valid) cudaGraphExecDestroy(ctx->gexec);
  if (ctx && ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  if (ctx && ctx->tev_made)
    for (int r = 0; r < TC_TIMING_RING; ++r)
      for (int p = 0; p <= TC_NPHASE; ++p) cudaEventDestroy(ctx->tev[r][p]);
  delete ctx;
  return TC_OK;
}

#define ST(c) ((cudaStream_t)(c))

// ---------------------------------------------------------------------------
// Typed implementations (T = storage type of the velocity fields)
// ---------------------------------------------------------------------------
__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, int n) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) b[e] = (float)a[e];
}

template <class T> static int set_state_impl(tc_ctx* c, const double* u, const double* v, const double* w, cudaStream_t s) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  dim3 blk(32, 8);
  dim3 gc((nx + 31) / 32, ny, (nz + 31) / 32), gf((nx + 31) / 32, ny, (nz + 1 + 31) / 32);
  T** S = (T**)c->st[c->cur];
  const double* base = nullptr;
  if (c->precision == TC_MIXED) {
    // base profile = per-plane mean of the incoming u; u is stored as u - U0[k]
    k_plane_mean_ref_u<<<nz, 256, 0, s>>>(u, nx, ny, nz, c->ubase_d);
    k_d2f<<<(nz + 255) / 256, 256, 0, s>>>(c->ubase_d, (float*)c->ubase_t, nz);
    base = c->ubase_d;
  }
  k_from_ref<T><<<gc, blk, 0, s>>>(u, S[0], FLD_U, nx, ny, nz, 1.0, base);
  k_from_ref<T><<<gc, blk, 0, s>>>(v, S[1], FLD_V, nx, ny, nz, 1.0, nullptr);
  k_from_ref<T><<<gf, blk, 0, s>>>(w, S[2], FLD_W, nx, ny, nz, 1.0, nullptr);
  TC_LAUNCHED();
  return TC_OK;
}

template <class T> static int to_ref(const tc_ctx* c, const T* in, double* out, int kind, cudaStream_t s,
                                     const double* base = nullptr) {
  int Xr, Zr;
  switch (kind) {
    case FLD_U: Xr = c->nx + 1; Zr = c->nz + 2; break;
    case FLD_V: Xr = c->nx + 2; Zr = c->nz + 2; break;
    case FLD_W: Xr = c->nx + 2; Zr = c->nz + 1; break;
    case FLD_P: Xr = c->nx + 2; Zr = c->nz + 2; break;
    default: Xr = c->nx; Zr = c->nz; break;
  }
  int Yr = (kind == FLD_U || kind == FLD_W || kind == FLD_P) ? c->ny + 2 : (kind == FLD_V ? c->ny + 1 : c->ny);
  dim3 grid((Xr + 31) / 32, Yr, (Zr + 31) / 32);
  k_to_ref<T><<<grid, dim3(32, 8), 0, s>>>(in, out, kind, c->nx, c->ny, c->nz, c->top_neumann, base);
  TC_LAUNCHED();
  return TC_OK;
}

static const double* ubase_of(const tc_ctx* c) { return c->precision == TC_MIXED ? c->ubase_d : nullptr; }

// Poisson solve of L p = scale * (div(u, v, w) or field): spectrum and p FP64.
// `field` and `p` may alias (the field is consumed by the first pass).
template <class T> static int poisson_impl(tc_ctx* c, const T* u, const T* v, const T* w, const double* field,
                                           double* p, double scale, cudaStream_t s) {
  Grid<T> g = make_grid<T>(c);
  const int nx = c->nx, ny = c->ny, nz = c->nz, nxh = c->nxh;
  cpx<double>* X = c->X;
  const size_t smx = ((size_t)2 * (c->JT / 2) * padded_len<double>(nx) + nx) * sizeof(cpx<double>);
  mark(c, TC_PH_FFTX, s);
  const bool xreg = xreg_ok(c);
  if (xreg)
    fftx_reg<T>(c, g, u, v, w, field, X, scale, s);
  else
    k_div_fftx<T><<<dim3(ny / c->JT, nz), 256, smx, s>>>(g, u, v, w, field, X, c->planx, c->twx_d, scale, c->JT);
  const int nrows = nxh * nz;
  const size_t smy = ((size_t)2 * c->RB * padded_len<double>(ny) + ny) * sizeof(cpx<double>);
  mark(c, TC_PH_FFTY, s);
  if (c->yz_on) {
    // one fused launch: the tri and inverse-y phases are empty
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = yz_config(c, at, s);
    PoissonTabs tb{c->k2x, c->k2y, c->cl, c->cr};
    if (c->yzr_ok) {
      cfg.blockDim = dim3(c->yzr_thr, 1, 1);
      cfg.dynamicSmemBytes = c->yzr_smem;
      int rc2 = TC_OK;
      for_each_n1(ny, [&](auto I) {
        constexpr int N1 = decltype(I)::value;
        cudaError_t e = c->yz_P <= 16
                            ? cudaLaunchKernelEx(&cfg, k_yz_solve_reg<N1, 16>, X, (const double*)c->tri_cpb, tb,
                                                 (const cpx<double>*)c->twy_d, nz, c->yz_P)
                            : cudaLaunchKernelEx(&cfg, k_yz_solve_reg<N1, 32>, X, (const double*)c->tri_cpb, tb,
                                                 (const cpx<double>*)c->twy_d, nz, c->yz_P);
        if (e != cudaSuccess) rc2 = fail(TC_ERR_CUDA, std::string("k_yz_solve_reg: ") + cudaGetErrorString(e));
      });
      if (rc2) return rc2;
    } else if (c->yz_P <= 16)
      TC_CUDA(cudaLaunchKernelEx(&cfg, k_yz_solve<16>, X, (const double*)c->tri_cpb, tb, c->plany,
                                 (const cpx<double>*)c->twy_d, ny, nz, c->yz_P, c->yz_FB));
    else
      TC_CUDA(cudaLaunchKernelEx(&cfg, k_yz_solve<32>, X, (const double*)c->tri_cpb, tb, c->plany,
                                 (const cpx<double>*)c->twy_d, ny, nz, c->yz_P, c->yz_FB));
    mark(c, TC_PH_TRI, s);
    mark(c, TC_PH_IFFTY, s);
    mark(c, TC_PH_IFFTX, s);
    if (xreg)
      ifftx_reg(c, X, p, s);
    else
      k_ifftx<<<dim3(ny / c->JT, nz), 256, smx, s>>>(X, p, nx, ny, nz, c->planx, c->twx_d, c->JT);
    TC_LAUNCHED();
    return TC_OK;
  }
  if (c->ys_on && c->tri_rden) {
    // two streaming passes: the tri phase is the forward pass's sweep
    ys_pass<false>(c, X, s);
    mark(c, TC_PH_TRI, s);
    mark(c, TC_PH_IFFTY, s);
    ys_pass<true>(c, X, s);
    mark(c, TC_PH_IFFTX, s);
    if (xreg)
      ifftx_reg(c, X, p, s);
    else
      k_ifftx<<<dim3(ny / c->JT, nz), 256, smx, s>>>(X, p, nx, ny, nz, c->planx, c->twx_d, c->JT);
    TC_LAUNCHED();
    return TC_OK;
  }
  const bool yreg = yreg_ok(c);
  if (yreg)
    ffty_reg<false>(c, X, nrows, s);
  else
    k_ffty<false><<<(nrows + c->RB - 1) / c->RB, 256, smy, s>>>(X, nrows, ny, c->plany, c->twy_d, c->RB);
  PoissonTabs tb{c->k2x, c->k2y, c->cl, c->cr};
  const int nmodes = nxh * ny;
  mark(c, TC_PH_TRI, s);
  if (c->tri_rden) {
    const int nb = (2 * nmodes + 63) / 64;
    if (nb <= c->tri16_blocks)
      k_tri_lu2<16><<<nb, 64, 0, s>>>(reinterpret_cast<double*>(X), c->tri_rden, c->tri_cp, tb, nxh, ny, nz);
    else
      k_tri_lu2<8><<<nb, 64, 0, s>>>(reinterpret_cast<double*>(X), c->tri_rden, c->tri_cp, tb, nxh, ny, nz);
  } else
    k_tri<<<(nmodes + c->tri_bt - 1) / c->tri_bt, c->tri_bt, (size_t)c->tri_bt * nz * 8, s>>>(X, tb, nxh, ny, nz);
  mark(c, TC_PH_IFFTY, s);
  if (yreg)
    ffty_reg<true>(c, X, nrows, s);
  else
    k_ffty<true><<<(nrows + c->RB - 1) / c->RB, 256, smy, s>>>(X, nrows, ny, c->plany, c->twy_d, c->RB);
  mark(c, TC_PH_IFFTX, s);
  if (xreg)
    ifftx_reg(c, X, p, s);
  else
    k_ifftx<<<dim3(ny / c->JT, nz), 256, smx, s>>>(X, p, nx, ny, nz, c->planx, c->twx_d, c->JT);
  TC_LAUNCHED();
  return TC_OK;
}

// The single-precision Poisson solve of a step: L dp = div(u**)/dt - L p_b,
// p_b = pf[pcur] the previous step's pressure, with the FP32 spectrum
// (L p_b into the dp buffer, x transform of the difference, the fused y / z /
// inverse-y slab kernel, inverse x transform into dp = c->p as FP32).
template <class T> static int poisson32_impl(tc_ctx* c, const T* u, const T* v, const T* w, double dt,
                                             cudaStream_t s) {
  if constexpr (sizeof(T) != 4) {
    return fail(TC_ERR_ARG, "the single-precision Poisson step needs a mixed-precision context");
  } else {
    Grid<float> g = make_grid<float>(c);
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    cpx<float>* Xf = reinterpret_cast<cpx<float>*>(c->X);
    float* dpf = reinterpret_cast<float*>(c->p);
    const double scale = 1.0 / (dt * (double)nx * (double)ny);
    mark(c, TC_PH_FFTX, s);
    k_base_lap<<<dim3((nx + 31) / 32, (ny + 7) / 8, nz), dim3(32, 8), 0, s>>>(
        c->pf[c->pcur], dpf, nx, ny, nz, 1.0 / (c->dx * c->dx), 1.0 / (c->dy * c->dy), c->cl, c->cr);
    for_each_n1(nx, [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      k_div_fftx_reg32<float, N1, XROWS><<<dim3(ny / XROWS, nz), xreg_threads<N1>(), fftx_reg_smem<N1>(), s>>>(
          g, u, v, w, Xf, c->twx_d, scale, dpf, 1.0 / ((double)nx * (double)ny));
    });
    mark(c, TC_PH_FFTY, s);
    for_each_yz32(ny, [&](auto I) {
      constexpr int K = decltype(I)::value;
      k_yz32<K><<<c->nxh, c->yz32_thr, c->yz32_smem, s>>>(Xf, c->rden32, c->cp32, c->tri_rden, c->tri_cp, c->cl,
                                                         c->twy32, nz, c->err);
    });
    mark(c, TC_PH_TRI, s);
    mark(c, TC_PH_IFFTY, s);
    mark(c, TC_PH_IFFTX, s);
    for_each_n1(nx, [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      k_ifftx_reg32<N1, XROWS><<<dim3(ny / XROWS, nz), xreg_threads<N1>(), ifftx_reg_smem<N1>(), s>>>(
          Xf, dpf, ny, nz, c->twx_d);
    });
    TC_LAUNCHED();
    return TC_OK;
  }
}

// Chunk length of the CN solve: 16 rows up to nz = 256 (at most 16 warps),
// 32 rows for deeper channels (nz <= 512).  The G/H tables follow it.
// CN tables of the context for time step dt and chunk length L: the build
// stages its work in shared memory where 17 nz doubles fit in the default
// 48 KB (nz <= 361), else it works in the tables themselves.
static void launch_cn_tables(tc_ctx* c, double dt, int L, cudaStream_t s) {
  const size_t sm = (size_t)17 * c->nz * sizeof(double);
  const bool staged = sm <= 48 * 1024;
  k_cn_tables<<<1, 32, staged ? sm : 0, s>>>(c->tab, c->dzf_d, c->dzc_d, c->nz, c->nu, dt, c->top_neumann, L,
                                             ubase_of(c), staged ? 1 : 0);
}

static int cn_len(const tc_ctx* c) {
  if (c->cn_L_force) return c->cn_L_force;
  return c->nz <= 256 ? 16 : 32;
}
static int cn_chunks(const tc_ctx* c) { return (c->nz + cn_len(c) - 1) / cn_len(c); }
template <class T> static size_t cn_smem(const tc_ctx* c) {
  const int vec = (cn_len(c) <= 16 && sizeof(T) == 4) ? 2 : 1;
  return (size_t)(9 * c->nz + 2 * cn_chunks(c) * 32 * vec) * 8;
}
template <class T> static void launch_cn(const tc_ctx* c, T* u, T* v, T* w, cudaStream_t s) {
  const int ncol = c->nx * c->ny;
  const dim3 blk(32, cn_chunks(c));
  const int Lr = cn_len(c);
  const size_t sm = cn_smem<T>(c);
  const double* ub = ubase_of(c);
  if (Lr <= 16) {
    constexpr int V = sizeof(T) == 4 ? 2 : 1;
    const dim3 grid((ncol / V + 31) / 32, 1, 3);
    if (Lr == 16)
      cn16_kernel<T, true>()<<<grid, blk, sm, s>>>(u, v, w, c->tab, ub, c->nx, c->ny, c->nz, Lr);
    else
      cn16_kernel<T, false>()<<<grid, blk, sm, s>>>(u, v, w, c->tab, ub, c->nx, c->ny, c->nz, Lr);
  } else {
    const dim3 grid((ncol + 31) / 32, 1, 3);
    if (Lr == 32)
      k_cn_solve<T, 32, 1, 512, true><<<grid, blk, sm, s>>>(u, v, w, c->tab, ub, c->nx, c->ny, c->nz, Lr);
    else
      k_cn_solve<T, 32, 1, 512, false><<<grid, blk, sm, s>>>(u, v, w, c->tab, ub, c->nx, c->ny, c->nz, Lr);
  }
}

static dim3 grid3(const tc_ctx* c, int planes) { return dim3((c->nx + 31) / 32, (c->ny + 7) / 8, planes); }

static double bulk_scale(const tc_ctx* c) { return c->dx * c->dy / (c->Lx * c->Ly * c->Lz); }

template <class T, class PS>
static int project_impl_ps(tc_ctx* c, T* const* S, const PS& ps, double dt, int update_forcing, cudaStream_t s) {
  Grid<T> g = make_grid<T>(c);
  BulkArgs ba{c->partials, c->ticket, c->scal, bulk_scale(c), c->U_bulk, dt, update_forcing};
  dim3 grd((c->nx / 2 + 31) / 32, (c->ny + 7) / 8, (c->nz + PROJ_PK - 1) / PROJ_PK);
  k_project_bulk<T, PS><<<grd, dim3(32, 8), 0, s>>>(g, S[0], S[1], S[2], ps, dt, c->dzf_d, ba);
  TC_LAUNCHED();
  return TC_OK;
}
template <class T> static int project_impl(tc_ctx* c, T* const* S, double dt, int update_forcing, cudaStream_t s) {
  return project_impl_ps<T, PSrc64>(c, S, PSrc64{c->p, nullptr}, dt, update_forcing, s);
}

template <class T> static int step_impl(tc_ctx* c, int scheme, double dt, cudaStream_t s) {
  Grid<T> g = make_grid<T>(c);
  const int nxt = c->cur ^ 1;
  T** A = (T**)c->st[c->cur];
  T** B = (T**)c->st[nxt];
  T** R = (T**)c->rh;
  dim3 blk(RHS_TX, rhs_ty<T>());
  dim3 grd((c->nx + RHS_TX - 1) / RHS_TX, (c->ny + rhs_ty<T>() - 1) / rhs_ty<T>(), (c->nz + 1 + rhs_kb<T>() - 1) / rhs_kb<T>());
  if (scheme == TC_IMEX && c->tab_dt != dt) {
    launch_cn_tables(c, dt, cn_len(c), s);
    c->tab_dt = dt;
  }
  // single-precision Poisson (IMEX): the increment over pf[pcur] once a base
  // exists and the warm-up steps after set_state are done.  Before that, and
  // for the explicit schemes, the FP64 solve, whose p (rounded) becomes the
  // base.
  const bool psp_now = psp_ready(c) && scheme == TC_IMEX;
  mark(c, TC_PH_RHS, s);
  if (c->rhs_tma_on) {
    if (scheme == TC_IMEX)
      launch_rhs_tma<T, false, UPD_AB2>(c, g, A, B, R, dt, c->have_hist, s);
    else if (scheme == TC_AB2)
      launch_rhs_tma<T, true, UPD_AB2>(c, g, A, B, R, dt, c->have_hist, s);
    else
      launch_rhs_tma<T, true, UPD_FE>(c, g, A, B, R, dt, 0, s);
  } else if (scheme == TC_IMEX)
    RhsKernel<T, false, UPD_AB2>::fn<<<grd, blk, 0, s>>>(g, A[0], A[1], A[2], B[0], B[1], B[2], R[0], R[1], R[2],
                                                         c->scal + SC_FORCING, (T)dt, c->have_hist);
  else if (scheme == TC_AB2)
    RhsKernel<T, true, UPD_AB2>::fn<<<grd, blk, 0, s>>>(g, A[0], A[1], A[2], B[0], B[1], B[2], R[0], R[1], R[2],
                                                        c->scal + SC_FORCING, (T)dt, c->have_hist);
  else
    RhsKernel<T, true, UPD_FE>::fn<<<grd, blk, 0, s>>>(g, A[0], A[1], A[2], B[0], B[1], B[2], R[0], R[1], R[2],
                                                       c->scal + SC_FORCING, (T)dt, 0);
  TC_LAUNCHED();
  if constexpr (sizeof(T) == 8) {
    if (c->body[0]) {  // R += F: q* += c F, r += F (FP64 contexts only)
      const double cq = (scheme == TC_FE || !c->have_hist) ? dt : 1.5 * dt;
      k_add_body<<<dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz + 1), dim3(32, 8), 0, s>>>(
          B[0], B[1], B[2], R[0], R[1], R[2], c->body[0], c->body[1], c->body[2], cq, scheme == TC_FE ? 0.0 : 1.0,
          c->nx, c->ny, c->nz);
      TC_LAUNCHED();
    }
  }
  mark(c, TC_PH_CN, s);
  if (scheme == TC_IMEX) {
    launch_cn<T>(c, B[0], B[1], B[2], s);
    TC_LAUNCHED();
  }
  int rc;
  if (psp_now)
    rc = poisson32_impl<T>(c, B[0], B[1], B[2], dt, s);
  else
    rc = poisson_impl<T>(c, B[0], B[1], B[2], nullptr, c->p, 1.0 / (dt * (double)c->nx * (double)c->ny), s);
  if (rc) return rc;
  mark(c, TC_PH_PROJ, s);
  if constexpr (sizeof(T) == 4) {
    if (psp_now)
      rc = project_impl_ps<T, PSrcInc>(c, B, PSrcInc{c->pf[c->pcur], reinterpret_cast<const float*>(c->p),
                                                       c->pf[c->pcur ^ 1]},
                                       dt, scheme != TC_FE, s);
    else
      rc = project_impl_ps<T, PSrc64>(c, B, PSrc64{c->p, c->psp_on ? c->pf[c->pcur ^ 1] : nullptr}, dt,
                                      scheme != TC_FE, s);
  } else {
    rc = project_impl<T>(c, B, dt, scheme != TC_FE, s);
  }
  if (rc) return rc;
  if constexpr (sizeof(T) == 8) {
    const dim3 ag((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz + 1);
    if (c->ke_acc || c->tape) {  // the adjoint hooks: one pass over the new state, one finishing block
      double* part = c->ke_acc ? c->ke_part : nullptr;
      k_step_hooks<<<ag, dim3(32, 8), 0, s>>>(B[0], B[1], B[2], c->dzf_d, c->dzc_d, c->ke_w, part, c->tape,
                                              c->tape_ctr, c->tape_slots, c->nx, c->ny, c->nz);
      k_step_hooks_finalize<<<1, 256, 0, s>>>(part, (int)(ag.x * ag.y * ag.z), c->ke_acc, c->ke_w,
                                              c->dx * c->dy / (c->Lx * c->Ly * c->Lz),
                                              c->tape ? c->tape_ctr : nullptr, c->tape_slots);
      TC_LAUNCHED();
    }
  }
  mark(c, TC_PH_FIN, s);
  mark(c, TC_NPHASE, s);
  if (c->timing) {
    c->t_head = (c->t_head + 1) % TC_TIMING_RING;
    if (c->t_count < TC_TIMING_RING) c->t_count++;
  }
  c->cur = nxt;
  if (scheme != TC_FE) c->have_hist = 1;
  if (c->psp_on) {
    c->pcur ^= 1;
    c->p_hist = 1;
  }
  c->p_f32 = psp_now;
  c->since_set++;
  return TC_OK;
}

template <class T> static int project_initial_impl(tc_ctx* c, cudaStream_t s) {
  T** A = (T**)c->st[c->cur];
  int rc = poisson_impl<T>(c, A[0], A[1], A[2], nullptr, c->p, 1.0 / ((double)c->nx * (double)c->ny), s);
  if (rc) return rc;
  return project_impl<T>(c, A, 1.0, 0, s);
}

template <class T> static int bulk_impl(tc_ctx* c, cudaStream_t s) {
  Grid<T> g = make_grid<T>(c);
  T** A = (T**)c->st[c->cur];
  dim3 grd = grid3(c, c->nz);
  k_bulk_partials<T><<<grd, dim3(32, 8), 0, s>>>(g, A[0], c->dzf_d, c->partials);
  k_bulk_finalize<<<1, 256, 0, s>>>(c->partials, grd.x * grd.y * grd.z, c->scal, bulk_scale(c), c->U_bulk, 1.0, 0);
  TC_LAUNCHED();
  return TC_OK;
}

template <class T> static int cfl_impl(tc_ctx* c, cudaStream_t s) {
  Grid<T> g = make_grid<T>(c);
  T** A = (T**)c->st[c->cur];
  dim3 grd = grid3(c, c->nz);
  k_cfl_partials<T><<<grd, dim3(32, 8), 0, s>>>(g, A[0], A[1], A[2], c->partials2);
  k_max_finalize<<<1, 256, 0, s>>>(c->partials2, grd.x * grd.y * grd.z, c->scal + SC_DTI);
  TC_LAUNCHED();
  return TC_OK;
}

template <class T> static int diag_impl(tc_ctx* c, cudaStream_t s) {
  Grid<T> g = make_grid<T>(c);
  T** A = (T**)c->st[c->cur];
  dim3 grd = grid3(c, c->nz);
  const int nb = grd.x * grd.y * grd.z;
  // nb = gx*gy*nz <= npart: one partials buffer each for the max and the flag
  if (c->p_f32)
    k_diag_partials<T, float><<<grd, dim3(32, 8), 0, s>>>(g, A[0], A[1], A[2], c->pf[c->pcur], c->partials2,
                                                          c->partials);
  else
    k_diag_partials<T><<<grd, dim3(32, 8), 0, s>>>(g, A[0], A[1], A[2], c->p, c->partials2, c->partials);
  k_max_finalize<<<1, 256, 0, s>>>(c->partials2, nb, c->scal + SC_MAXDIV);
  k_max_finalize<<<1, 256, 0, s>>>(c->partials, nb, c->scal + SC_NONFINITE);
  k_utau_sums<T><<<2, 256, 0, s>>>(g, A[0], c->scal);
  TC_LAUNCHED();
  return TC_OK;
}

template <class T> static int stats_impl(tc_ctx* c, cudaStream_t s) {
  T** A = (T**)c->st[c->cur];
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  k_stats_prof<T><<<nz, 256, 0, s>>>(A[0], A[1], A[2], nx, ny, nz, ubase_of(c), c->st_prof, c->st_means);
  k_stats_fill<T><<<(nx * ny + 255) / 256, 256, 0, s>>>(A[0], A[1], A[2], nx, ny, nz, c->k_bot - 1, c->k_top - 1,
                                                        ubase_of(c), c->st_means, c->st_S);
  const int nrows = 3 * ny;
  k_fft_rows_d<false><<<(nrows + c->stats_RB - 1) / c->stats_RB, 256,
                        ((size_t)2 * c->stats_RB * padded_len<double>(nx) + nx) * 16, s>>>(
      c->st_S, nrows, nx, c->planx, c->twx_d, c->stats_RB);
  const int bpp = (nx + c->stats_CB - 1) / c->stats_CB;
  k_fft_cols<false><<<3 * bpp, 256, ((size_t)2 * c->stats_CB * padded_len<double>(ny) + ny) * 16, s>>>(c->st_S, nx, ny, nx, (size_t)nx * ny,
                                                                          c->plany, c->twy_d, c->stats_CB);
  const int nspec = (nx / 2) * (ny / 2);
  k_stats_spec<<<(nspec + 127) / 128, 128, 0, s>>>(c->st_S, nx, ny, c->st_spec);
  TC_LAUNCHED();
  return TC_OK;
}

template <class T> static int rhs_hook_impl(tc_ctx* c, int full, double* ru, double* rv, double* rw, cudaStream_t s) {
  Grid<T> g = make_grid<T>(c);
  T** A = (T**)c->st[c->cur];
  T** B = (T**)c->st[c->cur ^ 1];  // scratch: the next buffer is free between steps
  const size_t ncell = (size_t)c->nx * c->ny * c->nz;
  cudaMemsetAsync(B[2], 0, ncell / c->nz * (c->nz + 1) * sizeof(T), s);
  dim3 grd((c->nx + RHS_TX - 1) / RHS_TX, (c->ny + rhs_ty<T>() - 1) / rhs_ty<T>(), (c->nz + 1 + rhs_kb<T>() - 1) / rhs_kb<T>());
  if (full)
    RhsKernel<T, true, UPD_RHS_ONLY>::fn<<<grd, dim3(RHS_TX, rhs_ty<T>()), 0, s>>>(g, A[0], A[1], A[2], nullptr, nullptr, nullptr,
                                                                   B[0], B[1], B[2], c->scal, (T)0, 0);
  else
    RhsKernel<T, false, UPD_RHS_ONLY>::fn<<<grd, dim3(RHS_TX, rhs_ty<T>()), 0, s>>>(g, A[0], A[1], A[2], nullptr, nullptr, nullptr,
                                                                    B[0], B[1], B[2], c->scal, (T)0, 0);
  TC_LAUNCHED();
  int rc;
  if ((rc = to_ref<T>(c, B[0], ru, FLD_U, s)) || (rc = to_ref<T>(c, B[1], rv, FLD_V, s)) ||
      (rc = to_ref<T>(c, B[2], rw, FLD_W, s)))
    return rc;
  return TC_OK;
}

// ---------------------------------------------------------------------------
// extern "C" entry points
// ---------------------------------------------------------------------------
#define DISPATCH(c, fn, ...) ((c)->tsz == 8 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

extern "C" int tc_set_state(tc_ctx* c, const double* u, const double* v, const double* w, double forcing, void* stream) {
  if (!c || !u || !v || !w) return fail(TC_ERR_ARG, "null argument");
  int rc = DISPATCH(c, set_state_impl, c, u, v, w, ST(stream));
  if (rc) return rc;
  TC_CUDA(cudaMemsetAsync(c->scal, 0, SC_COUNT * 8, ST(stream)));
  rc = tc_set_forcing(c, forcing, stream);
  if (rc) return rc;
  TC_CUDA(cudaMemsetAsync(c->p, 0, (size_t)c->nx * c->ny * c->nz * 8, ST(stream)));
  c->have_hist = 0;
  c->state_set = 1;
  c->p_hist = 0;   // no pressure base for a single-precision solve yet
  c->p_f32 = 0;
  c->since_set = 0;
  if (c->precision == TC_MIXED) c->tab_dt = -1.0;  // the CN tables carry the new base profile
  return TC_OK;
}

extern "C" int tc_set_forcing(tc_ctx* c, double forcing, void* stream) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  // a one-element H2D copy from a host stack value must complete before return
  TC_CUDA(cudaMemcpyAsync(c->scal + SC_FORCING, &forcing, 8, cudaMemcpyHostToDevice, ST(stream)));
  TC_CUDA(cudaStreamSynchronize(ST(stream)));
  return TC_OK;
}

template <class T> static int get_state_impl(tc_ctx* c, double* u, double* v, double* w, double* p, cudaStream_t s) {
  int rc = TC_OK;
  T** A = (T**)c->st[c->cur];
  if (u && (rc = to_ref<T>(c, A[0], u, FLD_U, s, ubase_of(c)))) return rc;
  if (v && (rc = to_ref<T>(c, A[1], v, FLD_V, s))) return rc;
  if (w && (rc = to_ref<T>(c, A[2], w, FLD_W, s))) return rc;
  if (p && c->p_f32 && (rc = to_ref<float>(c, c->pf[c->pcur], p, FLD_P, s))) return rc;
  if (p && !c->p_f32 && (rc = to_ref<double>(c, c->p, p, FLD_P, s))) return rc;
  return TC_OK;
}

extern "C" int tc_get_state(tc_ctx* c, double* u, double* v, double* w, double* p, void* stream) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  return DISPATCH(c, get_state_impl, c, u, v, w, p, ST(stream));
}

template <class T> static int get_hist_impl(tc_ctx* c, double* ru, double* rv, double* rw, cudaStream_t s) {
  int rc;
  T** R = (T**)c->rh;
  if (ru && (rc = to_ref<T>(c, R[0], ru, FLD_U, s))) return rc;
  if (rv && (rc = to_ref<T>(c, R[1], rv, FLD_V, s))) return rc;
  if (rw && (rc = to_ref<T>(c, R[2], rw, FLD_W, s))) return rc;
  return TC_OK;
}

template <class T> static int set_hist_impl(tc_ctx* c, const double* ru, const double* rv, const double* rw, cudaStream_t s) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  dim3 blk(32, 8);
  dim3 gc((nx + 31) / 32, ny, (nz + 31) / 32), gf((nx + 31) / 32, ny, (nz + 1 + 31) / 32);
  T** R = (T**)c->rh;
  k_from_ref<T><<<gc, blk, 0, s>>>(ru, R[0], FLD_U, nx, ny, nz, 1.0, nullptr);
  k_from_ref<T><<<gc, blk, 0, s>>>(rv, R[1], FLD_V, nx, ny, nz, 1.0, nullptr);
  k_from_ref<T><<<gf, blk, 0, s>>>(rw, R[2], FLD_W, nx, ny, nz, 1.0, nullptr);
  TC_LAUNCHED();
  return TC_OK;
}

extern "C" int tc_get_history(tc_ctx* c, double* ru, double* rv, double* rw, void* stream) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (!c->have_hist) return fail(TC_ERR_STATE, "no AB2 history yet");
  return DISPATCH(c, get_hist_impl, c, ru, rv, rw, ST(stream));
}

extern "C" int tc_set_history(tc_ctx* c, const double* ru, const double* rv, const double* rw, void* stream) {
  if (!c || !ru || !rv || !rw) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "set the state first");
  int rc = DISPATCH(c, set_hist_impl, c, ru, rv, rw, ST(stream));
  if (rc) return rc;
  c->have_hist = 1;
  return TC_OK;
}

// Capture two consecutive steps (the state buffers swap once per step, so a
// pair returns to the same buffers) into an executable graph.
static int build_graph(tc_ctx* c, int scheme, double dt) {
  if (c->g_valid) {
    cudaGraphExecDestroy(c->gexec);
    c->g_valid = 0;
  }
  if (!c->cap_stream) TC_CUDA(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  const int cur0 = c->cur, hist0 = c->have_hist;
  const int pcur0 = c->pcur, phist0 = c->p_hist, pf320 = c->p_f32, since0 = c->since_set;
  const int psp0 = psp_ready(c);
  TC_CUDA(cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal));
  int rc = TC_OK;
  for (int q = 0; q < 2 && rc == TC_OK; ++q) rc = DISPATCH(c, step_impl, c, scheme, dt, c->cap_stream);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->cap_stream, &graph);
  c->cur = cur0;  // capture launched nothing: restore the host-side state
  c->have_hist = hist0;
  c->pcur = pcur0; c->p_hist = phist0; c->p_f32 = pf320; c->since_set = since0;
  if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
  if (e != cudaSuccess) return fail(TC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&c->gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(TC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  c->g_valid = 1; c->g_scheme = scheme; c->g_dt = dt; c->g_cur = cur0;
  c->g_pcur = pcur0; c->g_psp = psp0;
  return TC_OK;
}

extern "C" int tc_step(tc_ctx* c, int scheme, double dt, int n_steps, void* stream) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  if (scheme != TC_IMEX && scheme != TC_AB2 && scheme != TC_FE) return fail(TC_ERR_ARG, "bad scheme");
  if (!(dt > 0) || n_steps < 0) return fail(TC_ERR_ARG, "dt must be > 0 and n_steps >= 0");
  int n = 0;
  // plain launches until the history exists and the CN tables match dt
  while (n < n_steps && (!c->have_hist || (scheme == TC_IMEX && c->tab_dt != dt) || c->timing || !c->graphs_on ||
                         (c->psp_on && !psp_ready(c)) || n_steps - n < 4)) {
    int rc = DISPATCH(c, step_impl, c, scheme, dt, ST(stream));
    if (rc) return rc;
    ++n;
  }
  if (n_steps - n >= 2) {
    if (!c->g_valid || c->g_scheme != scheme || c->g_dt != dt || c->g_cur != c->cur || c->g_pcur != c->pcur ||
        c->g_psp != (int)psp_ready(c)) {
      int rc = build_graph(c, scheme, dt);
      if (rc) return rc;
    }
    for (; n + 2 <= n_steps; n += 2) {
      TC_CUDA(cudaGraphLaunch(c->gexec, ST(stream)));
      c->since_set += 2;
    }
  }
  for (; n < n_steps; ++n) {
    int rc = DISPATCH(c, step_impl, c, scheme, dt, ST(stream));
    if (rc) return rc;
  }
  return TC_OK;
}

extern "C" int tc_use_graphs(tc_ctx* c, int on) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  c->graphs_on = on ? 1 : 0;
  return TC_OK;
}

extern "C" int tc_use_fused_poisson(tc_ctx* c, int on) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (on < 0 || on > 2) return fail(TC_ERR_ARG, "mode 0 .. 2");
  if (on == 1 && !c->yz_ok) return fail(TC_ERR_SIZE, "fused y/z Poisson kernel not launchable for this grid");
  if (on == 2 && !c->ys_ok) return fail(TC_ERR_SIZE, "streamed y/z Poisson passes not available for this grid");
  const int yz = on == 1, ys = on == 2;
  if (yz != c->yz_on || ys != c->ys_on) {
    c->yz_on = yz;
    c->ys_on = ys;
    if (c->g_valid) {  // the captured steps hold the other path
      cudaGraphExecDestroy(c->gexec);
      c->g_valid = 0;
    }
  }
  return TC_OK;
}

extern "C" int tc_use_bulk_ffty(tc_ctx* c, int on) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (on && !c->ybulk_ok) return fail(TC_ERR_SIZE, "bulk-staged y transforms not available for this grid");
  if ((on ? 1 : 0) != c->ybulk_on) {
    c->ybulk_on = on ? 1 : 0;
    if (c->g_valid) {  // the captured steps hold the other kernel
      cudaGraphExecDestroy(c->gexec);
      c->g_valid = 0;
    }
  }
  return TC_OK;
}

extern "C" int tc_use_tma_rhs(tc_ctx* c, int on) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (on < 0 || on > 6) return fail(TC_ERR_ARG, "mode 0 .. 6");
  if (on && on != c->rhs_tma_mode) {
    const int rc = (c->tsz == 8) ? rhs_tma_setup<double>(c, on) : rhs_tma_setup<float>(c, on);
    if (rc) return rc;
  }
  if (on && !c->rhs_tma_ok) return fail(TC_ERR_SIZE, "tensor-copy RHS not available for this grid");
  c->rhs_tma_on = on ? 1 : 0;
  if (c->g_valid) {  // the captured steps may hold the other kernel
    cudaGraphExecDestroy(c->gexec);
    c->g_valid = 0;
  }
  return TC_OK;
}

extern "C" int tc_use_fp32_poisson(tc_ctx* c, int on, int warm_steps) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (warm_steps < 0) return fail(TC_ERR_ARG, "warm_steps must be >= 0");
  if (on && c->precision != TC_MIXED) return fail(TC_ERR_ARG, "the single-precision Poisson step needs TC_MIXED");
  if (on && !c->psp_ok)
    return fail(TC_ERR_SIZE, "single-precision Poisson step not available for this grid (register-transform nx, "
                             "ny = 16 K with K <= 24, and a kx slab of ny * nz * 8 bytes within shared memory)");
  const int was = c->psp_on;
  c->psp_on = on ? 1 : 0;
  c->psp_warm = warm_steps;
  if (c->psp_on && !was) c->p_hist = 0;  // the ring holds no base yet
  if (c->g_valid) {  // the captured steps hold the other path
    cudaGraphExecDestroy(c->gexec);
    c->g_valid = 0;
  }
  return TC_OK;
}

extern "C" int tc_project_initial(tc_ctx* c, void* stream) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  c->p_hist = 0;  // the dt = 1 pressure of this projection is no base for a step
  c->p_f32 = 0;
  return DISPATCH(c, project_initial_impl, c, ST(stream));
}

extern "C" int tc_scalars(tc_ctx* c, double** dev_ptr) {
  if (!c || !dev_ptr) return fail(TC_ERR_ARG, "null argument");
  *dev_ptr = c->scal;
  return TC_OK;
}

static int read_scal(tc_ctx* c, double* host, cudaStream_t s) {
  TC_CUDA(cudaMemcpyAsync(host, c->scal, SC_COUNT * 8, cudaMemcpyDeviceToHost, s));
  TC_CUDA(cudaStreamSynchronize(s));
  return TC_OK;
}

extern "C" int tc_bulk_velocity(tc_ctx* c, double* out, void* stream) {
  if (!c || !out) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  int rc = DISPATCH(c, bulk_impl, c, ST(stream));
  if (rc) return rc;
  double h[SC_COUNT];
  if ((rc = read_scal(c, h, ST(stream)))) return rc;
  *out = h[SC_UBULK];
  return TC_OK;
}

extern "C" int tc_cfl(tc_ctx* c, double* dti, void* stream) {
  if (!c || !dti) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  int rc = DISPATCH(c, cfl_impl, c, ST(stream));
  if (rc) return rc;
  double h[SC_COUNT];
  if ((rc = read_scal(c, h, ST(stream)))) return rc;
  *dti = h[SC_DTI];
  return TC_OK;
}

extern "C" int tc_diagnostics(tc_ctx* c, double* out, void* stream) {
  if (!c || !out) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  int rc = DISPATCH(c, diag_impl, c, ST(stream));
  if (rc) return rc;
  double h[SC_COUNT];
  if ((rc = read_scal(c, h, ST(stream)))) return rc;
  // u_tau (utils.py:176-204): first cell centre z_c[1] = dz_f[0]/2
  const double dist = 0.5 * c->dzf[0];
  const double tb = c->nu * h[SC_UTAU_BOT] / dist;
  const double ut_b = std::sqrt(std::fabs(tb));
  double ut = ut_b;
  if (!c->top_neumann) {
    const double tt = c->nu * h[SC_UTAU_TOP] / dist;
    ut = 0.5 * (ut_b + std::sqrt(std::fabs(tt)));
  }
  out[0] = h[SC_MAXDIV];
  out[1] = ut;
  out[2] = h[SC_UBULK];
  out[3] = h[SC_FORCING];
  out[4] = h[SC_NONFINITE];
  return TC_OK;
}

template <class T>
__global__ void k_div_field(Grid<T> g, const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ w,
                            double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int nx = g.nx, ny = g.ny;
  const size_t o = pidx(k, j, i, ny, nx);
  out[o] = ((double)u[o] - (double)u[pidx(k, j, wrap(i - 1, nx), ny, nx)]) * (double)g.idx +
           ((double)v[o] - (double)v[pidx(k, wrap(j - 1, ny), i, ny, nx)]) * (double)g.idy +
           ((double)w[pidx(k + 1, j, i, ny, nx)] - (double)w[o]) * (double)g.idzf[k];
}

// The next state buffer is free between steps; its u, v, w regions are
// carved back to back, so its start holds nx*ny*nz doubles in either precision.
static double* scratch_field(tc_ctx* c) { return (double*)c->st[c->cur ^ 1][0]; }

template <class T> static int divergence_impl(tc_ctx* c, double* div, cudaStream_t s) {
  T** A = (T**)c->st[c->cur];
  Grid<T> g = make_grid<T>(c);
  double* f = scratch_field(c);
  k_div_field<T><<<grid3(c, c->nz), dim3(32, 8), 0, s>>>(g, A[0], A[1], A[2], f);
  TC_LAUNCHED();
  return to_ref<double>(c, f, div, FLD_CELL, s);
}

extern "C" int tc_divergence(tc_ctx* c, double* div, void* stream) {
  if (!c || !div) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  return DISPATCH(c, divergence_impl, c, div, ST(stream));
}

extern "C" int tc_explicit_rhs(tc_ctx* c, int full, double* ru, double* rv, double* rw, void* stream) {
  if (!c || !ru || !rv || !rw) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  return DISPATCH(c, rhs_hook_impl, c, full, ru, rv, rw, ST(stream));
}

template <class T> static int cn_hook_impl(tc_ctx* c, double dt, cudaStream_t s) {
  T** A = (T**)c->st[c->cur];
  if (c->tab_dt != dt) {
    launch_cn_tables(c, dt, cn_len(c), s);
    c->tab_dt = dt;
  }
  launch_cn<T>(c, A[0], A[1], A[2], s);
  TC_LAUNCHED();
  return TC_OK;
}

extern "C" int tc_implicit_diffusion(tc_ctx* c, double dt, void* stream) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  if (!(dt > 0)) return fail(TC_ERR_ARG, "dt must be > 0");
  return DISPATCH(c, cn_hook_impl, c, dt, ST(stream));
}

template <class T> static int poisson_hook_impl(tc_ctx* c, const double* rhs, double* p, cudaStream_t s) {
  // rhs -> internal cell layout in the free state buffer, solve in place
  // (the solve consumes the field before it writes p), write out with ghosts.
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  double* f = scratch_field(c);
  k_from_ref<double><<<dim3((nx + 31) / 32, ny, (nz + 31) / 32), dim3(32, 8), 0, s>>>(rhs, f, FLD_CELL, nx, ny, nz,
                                                                                       1.0, nullptr);
  TC_LAUNCHED();
  int rc = poisson_impl<T>(c, nullptr, nullptr, nullptr, f, f, 1.0 / ((double)nx * (double)ny), s);
  if (rc) return rc;
  return to_ref<double>(c, f, p, FLD_P, s);
}

extern "C" int tc_poisson_solve(tc_ctx* c, const double* rhs, double* p, void* stream) {
  if (!c || !rhs || !p) return fail(TC_ERR_ARG, "null argument");
  return DISPATCH(c, poisson_hook_impl, c, rhs, p, ST(stream));
}

__global__ void k_p_from_ref(const double* __restrict__ ref, double* __restrict__ out, int nx, int ny, int nz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
  if (i >= nx || j >= ny || k >= nz) return;
  out[pidx(k, j, i, ny, nx)] = ref[((size_t)(i + 1) * (ny + 2) + (j + 1)) * (nz + 2) + (k + 1)];
}

template <class T> static int project_hook_impl(tc_ctx* c, const double* p, double dt, cudaStream_t s) {
  k_p_from_ref<<<grid3(c, c->nz), dim3(32, 8), 0, s>>>(p, c->p, c->nx, c->ny, c->nz);
  TC_LAUNCHED();
  return project_impl<T>(c, (T* const*)c->st[c->cur], dt, 0, s);
}

extern "C" int tc_project(tc_ctx* c, const double* p, double dt, void* stream) {
  if (!c || !p) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  c->p_f32 = 0;  // the given p (in the FP64 buffer) is the current one
  return DISPATCH(c, project_hook_impl, c, p, dt, ST(stream));
}

extern "C" int tc_stats_init(tc_ctx* c, const double* z_c, double Re_tau_target, double z_plus_target, int* k_bot,
                             int* k_top) {
  if (!c || !z_c) return fail(TC_ERR_ARG, "null argument");
  // turbstats.py:52-69
  const double u_tau_target = Re_tau_target * c->nu / (c->Lz / 2.0);
  const double zt = z_plus_target * c->nu / u_tau_target;
  int kb = 0, kt = 0;
  double bb = INFINITY, bt = INFINITY;
  for (int k = 0; k < c->nz; ++k) {
    double z = z_c[k + 1];
    double db = std::fabs(z - zt), dt_ = std::fabs(z - (c->Lz - zt));
    if (db < bb) { bb = db; kb = k; }
    if (dt_ < bt) { bt = dt_; kt = k; }
  }
  c->k_bot = kb + 1;
  c->k_top = kt + 1;
  if (k_bot) *k_bot = c->k_bot;
  if (k_top) *k_top = c->k_top;
  TC_CUDA(cudaMemset(c->st_prof, 0, 5 * c->nz * 8));
  TC_CUDA(cudaMemset(c->st_spec, 0, (size_t)4 * (c->nx / 2) * (c->ny / 2) * 8));
  TC_CUDA(cudaDeviceSynchronize());
  c->n_samples = 0;
  c->stats_ready = 1;
  return TC_OK;
}

extern "C" int tc_stats_accumulate(tc_ctx* c, void* stream) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (!c->stats_ready) return fail(TC_ERR_STATE, "call tc_stats_init first");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  int rc = DISPATCH(c, stats_impl, c, ST(stream));
  if (rc) return rc;
  c->n_samples++;
  return TC_OK;
}

extern "C" int tc_stats_read(tc_ctx* c, double* prof, double* spec, int* n_samples) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (!c->stats_ready) return fail(TC_ERR_STATE, "call tc_stats_init first");
  TC_CUDA(cudaDeviceSynchronize());
  if (prof) TC_CUDA(cudaMemcpy(prof, c->st_prof, 5 * c->nz * 8, cudaMemcpyDeviceToHost));
  if (spec) TC_CUDA(cudaMemcpy(spec, c->st_spec, (size_t)4 * (c->nx / 2) * (c->ny / 2) * 8, cudaMemcpyDeviceToHost));
  if (n_samples) *n_samples = c->n_samples;
  return TC_OK;
}

extern "C" int tc_stats_write(tc_ctx* c, const double* prof, const double* spec, int n_samples) {
  if (!c || !prof || !spec || n_samples < 0) return fail(TC_ERR_ARG, "bad argument");
  if (!c->stats_ready) return fail(TC_ERR_STATE, "call tc_stats_init first");
  TC_CUDA(cudaDeviceSynchronize());
  TC_CUDA(cudaMemcpy(c->st_prof, prof, 5 * c->nz * 8, cudaMemcpyHostToDevice));
  TC_CUDA(cudaMemcpy(c->st_spec, spec, (size_t)4 * (c->nx / 2) * (c->ny / 2) * 8, cudaMemcpyHostToDevice));
  c->n_samples = n_samples;
  return TC_OK;
}

extern "C" int tc_timing_enable(tc_ctx* c, int on) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (on && !c->tev_made) {
    for (int r = 0; r < TC_TIMING_RING; ++r)
      for (int p = 0; p <= TC_NPHASE; ++p) TC_CUDA(cudaEventCreate(&c->tev[r][p]));
    c->tev_made = 1;
  }
  c->timing = on ? 1 : 0;
  c->t_head = 0;
  c->t_count = 0;
  return TC_OK;
}

extern "C" int tc_timing_read(tc_ctx* c, double* ms, int* n_steps) {
  if (!c || !ms) return fail(TC_ERR_ARG, "null argument");
  for (int p = 0; p < TC_NPHASE; ++p) ms[p] = 0.0;
  if (n_steps) *n_steps = 0;
  if (!c->tev_made) return TC_OK;
  TC_CUDA(cudaDeviceSynchronize());
  for (int q = 0; q < c->t_count; ++q) {
    int r = (c->t_head - 1 - q + 2 * TC_TIMING_RING) % TC_TIMING_RING;
    int prev = -1;
    // phases that did not run in a step (CN outside IMEX) have no event: walk
    // the recorded boundaries in order and charge each interval to its start
    for (int p = 0; p <= TC_NPHASE; ++p) {
      if (cudaEventQuery(c->tev[r][p]) != cudaSuccess) continue;
      if (prev >= 0) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, c->tev[r][prev], c->tev[r][p]) == cudaSuccess) ms[prev] += t;
      }
      prev = p;
    }
  }
  cudaGetLastError();
  if (n_steps) *n_steps = c->t_count;
  c->t_count = 0;
  c->t_head = 0;
  return TC_OK;
}

extern "C" int tc_error(tc_ctx* c, int* code) {
  if (!c || !code) return fail(TC_ERR_ARG, "null argument");
  TC_CUDA(cudaDeviceSynchronize());
  TC_CUDA(cudaMemcpy(code, c->err, sizeof(int), cudaMemcpyDeviceToHost));
  TC_CUDA(cudaMemset(c->err, 0, sizeof(int)));
  return TC_OK;
}

extern "C" int tc_bounds_error(int* flag, int* where) {
  if (!flag || !where) return fail(TC_ERR_ARG, "null argument");
#ifdef TC_BOUNDS_CHECK
  TC_CUDA(cudaDeviceSynchronize());
  unsigned int w = 0;
  int at = 0;
  TC_CUDA(cudaMemcpyFromSymbol(&w, tc::tc_bounds_word, sizeof(w)));
  TC_CUDA(cudaMemcpyFromSymbol(&at, tc::tc_bounds_where, sizeof(at)));
  const unsigned int zw = 0;
  const int za = 0;
  TC_CUDA(cudaMemcpyToSymbol(tc::tc_bounds_word, &zw, sizeof(zw)));
  TC_CUDA(cudaMemcpyToSymbol(tc::tc_bounds_where, &za, sizeof(za)));
  *flag = w ? 1 : 0;
  *where = at;
#else
  *flag = -1;
  *where = 0;
#endif
  return TC_OK;
}

// ---------------------------------------------------------------------------
// Poisson solve that allocates nothing (tc_poisson_solve_noalloc).
//
// Some callers cannot hand this library a workspace: a host application whose
// device memory is owned by its own pool manager and forbids direct
// cudaMalloc / cudaFree, or a latency-critical loop that must not pay the
// device-wide synchronisation a cudaMalloc / cudaFree can cause.  For them the
// spectral intermediate and the small tables live in one fixed-size array in
// device global memory that the library owns for the life of the process.
// ---------------------------------------------------------------------------
#include <cuda.h>  // CUcontext and CUresult only: the driver calls are looked up at run time
#include <mutex>

#define TC_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define TC_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char tc_noalloc_scratch[TC_NOALLOC_SCRATCH_BYTES];

// Register-FFT lengths 16 N1 (rowfft_supported) and an index per N1 for the
// per-context occupancy cache below.
static constexpr int kNoallocN1[12] = {4, 6, 8, 9, 12, 16, 18, 24, 32, 36, 48, 64};
static int noalloc_n1_index(int n1) {
  for (int e = 0; e < 12; ++e)
    if (kNoallocN1[e] == n1) return e;
  return -1;
}
template <int E = 0, class F> static void for_all_n1(F&& f) {
  if constexpr (E < 12) {
    f(std::integral_constant<int, kNoallocN1[E]>{}, E);
    for_all_n1<E + 1>(f);
  }
}

// What the set-up of a device's context leaves for later calls: the context
// it ran in (a unique id, so that a context created after cudaDeviceReset is
// set up again), the SM count and the resident-block counts of the
// register y transform (per length) and of the 16-level z solve.
struct NoallocDev {
  unsigned long long ctx_id;
  int nsm;
  int ffty_nb[12];
  int tri16_nb;
};
static std::mutex g_noalloc_mu;
static NoallocDev g_noalloc_dev[TC_NOALLOC_MAX_DEVICES];

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (driver calls found
// through the runtime, so the library needs no link-time libcuda).
static int noalloc_ctx_id(unsigned long long* id) {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  if (!get_cur || !get_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0, q1;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1) {
      cudaGetLastError();
      return fail(TC_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId not found");
    }
    get_cur = (CtxGetCurrentFn)f0;
    get_id = (CtxGetIdFn)f1;
  }
  CUcontext ctx = nullptr;
  if (get_cur(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS)
    return fail(TC_ERR_CUDA, "no current CUDA context");
  return TC_OK;
}

// The host-side name tc_noalloc_scratch is not a device address: its
// address is looked up on every call (a cheap query in the current context).
// Kernel attributes and occupancy figures are set up once per context, in the
// first call made in it.
static int noalloc_setup(int dev, unsigned char** out, NoallocDev* info) {
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, tc_noalloc_scratch);
  if (e != cudaSuccess) return fail(TC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  unsigned long long id = 0;
  int rc = noalloc_ctx_id(&id);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoallocDev& d = g_noalloc_dev[dev];
  if (d.ctx_id != id) {
    NoallocDev n{};
    if ((rc = set_smem_attrs<double>(nullptr))) return rc;
    TC_CUDA(cudaDeviceGetAttribute(&n.nsm, cudaDevAttrMultiProcessorCount, dev));
    for_all_n1([&](auto I, int idx) {
      constexpr int N1 = decltype(I)::value;
      int nb = 0;
      if (cudaFuncSetAttribute(k_div_fftx_reg<double, N1, XROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)fftx_reg_smem<N1>()) != cudaSuccess ||
          cudaFuncSetAttribute(k_ifftx_reg<N1, XROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ifftx_reg_smem<N1>()) != cudaSuccess ||
          cudaFuncSetAttribute(k_ffty_reg<N1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ffty_reg_smem<N1>()) != cudaSuccess ||
          cudaFuncSetAttribute(k_ffty_reg<N1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ffty_reg_smem<N1>()) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ffty_reg<N1, false>, 128, ffty_reg_smem<N1>()) !=
              cudaSuccess)
        rc = fail(TC_ERR_CUDA, "register FFT attributes");
      n.ffty_nb[idx] = nb;
    });
    if (rc) return rc;
    TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n.tri16_nb, k_tri_lu2<16>, 64, 0));
    n.ctx_id = id;
    d = n;
  }
  *info = d;
  *out = (unsigned char*)ptr;
  return TC_OK;
}

// A caller's array must be device (or managed) memory of the current device:
// a host pointer handed to the kernels would fault instead of failing here.
static int noalloc_check_ptr(const void* p, int dev, const char* name) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return fail(TC_ERR_ARG, std::string(name) + ": not a CUDA pointer");
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return fail(TC_ERR_ARG, std::string(name) + " must be device memory (got host or unregistered memory)");
  if (a.type == cudaMemoryTypeDevice && a.device != dev)
    return fail(TC_ERR_ARG, std::string(name) + " belongs to another device");
  return TC_OK;
}

// Poisson tables from the grid (same definitions as tc_create's host tables:
// projection_fft.py:26-82), computed on the device so that nothing is copied
// from host memory.
__global__ void k_noalloc_tables(int nx, int ny, int nz, double dx, double dy, const double* __restrict__ dzf,
                                 const double* __restrict__ dzc, double* k2x, double* k2y, double* cl, double* cr,
                                 cpx<double>* twx, cpx<double>* twy) {
  const int nxh = nx / 2 + 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nxh + ny + nz + nx + ny; e += gridDim.x * blockDim.x) {
    int m = e;
    if (m < nxh) {
      double s = sinpi((double)m / (double)nx) * (2.0 / dx);
      k2x[m] = s * s;
      continue;
    }
    m -= nxh;
    if (m < ny) {
      double s = sinpi((double)m / (double)ny) * (2.0 / dy);
      k2y[m] = s * s;
      continue;
    }
    m -= ny;
    if (m < nz) {
      cl[m] = 1.0 / (dzc[m] * dzf[m]);
      cr[m] = 1.0 / (dzc[m + 1] * dzf[m]);
      continue;
    }
    m -= nz;
    if (m < nx) {
      double s, c;
      sincospi(-2.0 * (double)m / (double)nx, &s, &c);
      twx[m] = cpx<double>{c, s};
      continue;
    }
    m -= nx;
    double s, c;
    sincospi(-2.0 * (double)m / (double)ny, &s, &c);
    twy[m] = cpx<double>{c, s};
  }
}

static size_t noalloc_bytes(int nx, int ny, int nz, size_t off[8]) {
  const size_t nxh = nx / 2 + 1;
  // field (rhs in, p out), spectrum, k2x, k2y, cl, cr, x and y twiddles
  const size_t sz[8] = {(size_t)nx * ny * nz * 8, nxh * nz * ny * 16, nxh * 8, (size_t)ny * 8,
                        (size_t)nz * 8, (size_t)nz * 8, (size_t)nx * 16, (size_t)ny * 16};
  size_t o = 0;
  for (int e = 0; e < 8; ++e) {
    o = (o + 255) & ~(size_t)255;
    off[e] = o;
    o += sz[e];
  }
  return o;
}

extern "C" int tc_poisson_solve_noalloc(int nx, int ny, int nz, double Lx, double Ly, const double* dz_f,
                                        const double* dz_c, const double* rhs, double* p, void* stream) {
  if (!dz_f || !dz_c || !rhs || !p) return fail(TC_ERR_ARG, "null argument");
  if (nx < 8 || ny < 8 || nz < 4 || (nx & 1) || (ny & 1) || nz > 800 || !(Lx > 0) || !(Ly > 0))
    return fail(TC_ERR_SIZE, "nx, ny even >= 8, 4 <= nz <= 800, Lx, Ly > 0 required");
  FftPlan a, b;
  if (!fft_make_plan(nx, &a) || !fft_make_plan(ny, &b) || nx > 4096 || ny > 4096)
    return fail(TC_ERR_SIZE, "nx and ny must factor into 2 and 3 only (<= 4096)");
  size_t off[8];
  const size_t need = noalloc_bytes(nx, ny, nz, off);
  if (need > TC_NOALLOC_SCRATCH_BYTES)
    return fail(TC_ERR_SIZE, "grid needs " + std::to_string(need) + " bytes of scratch; the static maximum is " +
                                 std::to_string((size_t)TC_NOALLOC_SCRATCH_BYTES) + " bytes");
  int dev = 0;
  TC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= TC_NOALLOC_MAX_DEVICES) return fail(TC_ERR_ARG, "device index out of range");
  int rc;
  if ((rc = noalloc_check_ptr(dz_f, dev, "dz_f")) || (rc = noalloc_check_ptr(dz_c, dev, "dz_c")) ||
      (rc = noalloc_check_ptr(rhs, dev, "rhs")) || (rc = noalloc_check_ptr(p, dev, "p")))
    return rc;
  unsigned char* base = nullptr;
  NoallocDev info{};
  if ((rc = noalloc_setup(dev, &base, &info))) return rc;
  cudaStream_t s = ST(stream);
  // a context view over the static scratch (launch shapes as tc_create picks them)
  tc_grid_desc g{};
  g.nx = nx; g.ny = ny; g.nz = nz; g.Lx = Lx; g.Ly = Ly; g.Lz = 1.0; g.nu = 1.0; g.precision = TC_FP64;
  tc_ctx c{};
  fill_basic(&c, &g);
  c.dev = dev;
  c.nsm = info.nsm;
  c.yreg_blocks = c.nsm;
  if (yreg_ok(&c)) {
    const int nb = info.ffty_nb[noalloc_n1_index(ny / 16)];
    if (nb > 0) c.yreg_blocks = nb * c.nsm;
  }
  c.tri16_blocks = info.tri16_nb * c.nsm;
  double* field = (double*)(base + off[0]);
  c.X = (cpx<double>*)(base + off[1]);
  c.k2x = (double*)(base + off[2]); c.k2y = (double*)(base + off[3]);
  c.cl = (double*)(base + off[4]); c.cr = (double*)(base + off[5]);
  c.twx_d = (cpx<double>*)(base + off[6]); c.twy_d = (cpx<double>*)(base + off[7]);
  const int ntab = c.nxh + ny + nz + nx + ny;
  k_noalloc_tables<<<(ntab + 255) / 256, 256, 0, s>>>(nx, ny, nz, c.dx, c.dy, dz_f, dz_c, c.k2x, c.k2y, c.cl, c.cr,
                                                     c.twx_d, c.twy_d);
  k_from_ref<double><<<dim3((nx + 31) / 32, ny, (nz + 31) / 32), dim3(32, 8), 0, s>>>(rhs, field, FLD_CELL, nx, ny,
                                                                                        nz, 1.0, nullptr);
  TC_LAUNCHED();
  // every pass overwrites what it reads next, so no buffer needs clearing;
  // the solve writes p over the consumed right-hand side
  rc = poisson_impl<double>(&c, nullptr, nullptr, nullptr, field, field, 1.0 / ((double)nx * (double)ny), s);
  if (rc) return rc;
  return to_ref<double>(&c, field, p, FLD_P, s);
}

// ===========================================================================
// Adjoint of the IMEX step (FP64 contexts).  Arrays are in the internal
// layout: u, v nz planes of nx*ny (x fastest), w nz+1 face planes (walls 0).
// ===========================================================================
static size_t adj_field(const tc_ctx* c) { return (size_t)(c->nz + 1) * c->nx * c->ny; }
static size_t adj_nblocks(const tc_ctx* c) {
  return (size_t)((c->nx + 31) / 32) * ((c->ny + 7) / 8) * (c->nz + 1);
}
// scratch: lambda_R (3 fields), A (3 fields), CN tables (12 nz + 1), partials
struct AdjScratch {
  double* R[3]; double* A[3]; double* tab; double* partials;
};
static size_t adj_scratch_doubles(const tc_ctx* c) { return 6 * adj_field(c) + 12 * (size_t)c->nz + 1 + adj_nblocks(c); }
static AdjScratch adj_carve(const tc_ctx* c, void* scratch) {
  AdjScratch a;
  double* p = (double*)scratch;
  const size_t f = adj_field(c);
  for (int q = 0; q < 3; ++q) a.R[q] = p + q * f;
  for (int q = 0; q < 3; ++q) a.A[q] = p + (3 + q) * f;
  a.tab = p + 6 * f;
  a.partials = a.tab + 12 * (size_t)c->nz + 1;
  return a;
}
static int adj_check(const tc_ctx* c, const void* scratch) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (c->precision != TC_FP64) return fail(TC_ERR_ARG, "the adjoint needs an FP64 context");
  if (scratch && ((uintptr_t)scratch & 15)) return fail(TC_ERR_WORKSPACE, "adjoint scratch must be 16-byte aligned");
  return TC_OK;
}
static dim3 adj_grid(const tc_ctx* c) { return dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz + 1); }

extern "C" int tc_adjoint_scratch_bytes(tc_ctx* c, size_t* bytes) {
  int rc = adj_check(c, nullptr);
  if (rc) return rc;
  if (!bytes) return fail(TC_ERR_ARG, "null bytes");
  *bytes = adj_scratch_doubles(c) * sizeof(double);
  return TC_OK;
}

extern "C" int tc_set_body_force(tc_ctx* c, const double* fu, const double* fv, const double* fw) {
  int rc = adj_check(c, nullptr);
  if (rc) return rc;
  if ((fu || fv || fw) && !(fu && fv && fw)) return fail(TC_ERR_ARG, "body force needs all three components or none");
  c->body[0] = fu; c->body[1] = fv; c->body[2] = fw;
  if (c->g_valid) {  // captured steps hold the previous forcing
    cudaGraphExecDestroy(c->gexec);
    c->g_valid = 0;
  }
  return TC_OK;
}

extern "C" int tc_internal_doubles(tc_ctx* c, size_t* n) {
  int rc = adj_check(c, nullptr);
  if (rc) return rc;
  if (!n) return fail(TC_ERR_ARG, "null n");
  *n = 6 * adj_field(c) + 1;
  return TC_OK;
}

// state record: u, v, w, r_u, r_v, r_w (each adj_field doubles, u/v padded
// with one zero plane), forcing.
extern "C" int tc_save_internal(tc_ctx* c, double* dst, int* have_hist, void* stream) {
  int rc = adj_check(c, nullptr);
  if (rc) return rc;
  if (!dst || !have_hist) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  cudaStream_t s = ST(stream);
  const size_t f = adj_field(c), pl = (size_t)c->nx * c->ny;
  for (int q = 0; q < 3; ++q) {
    const size_t n = (q < 2 ? (size_t)c->nz : (size_t)c->nz + 1) * pl;
    TC_CUDA(cudaMemcpyAsync(dst + q * f, c->st[c->cur][q], n * 8, cudaMemcpyDeviceToDevice, s));
    if (q < 2) TC_CUDA(cudaMemsetAsync(dst + q * f + n, 0, pl * 8, s));
    TC_CUDA(cudaMemcpyAsync(dst + (3 + q) * f, c->rh[q], n * 8, cudaMemcpyDeviceToDevice, s));
    if (q < 2) TC_CUDA(cudaMemsetAsync(dst + (3 + q) * f + n, 0, pl * 8, s));
  }
  TC_CUDA(cudaMemcpyAsync(dst + 6 * f, c->scal + SC_FORCING, 8, cudaMemcpyDeviceToDevice, s));
  *have_hist = c->have_hist;
  return TC_OK;
}

extern "C" int tc_load_internal(tc_ctx* c, const double* src, int have_hist, void* stream) {
  int rc = adj_check(c, nullptr);
  if (rc) return rc;
  if (!src) return fail(TC_ERR_ARG, "null argument");
  cudaStream_t s = ST(stream);
  const size_t f = adj_field(c), pl = (size_t)c->nx * c->ny;
  for (int q = 0; q < 3; ++q) {
    const size_t n = (q < 2 ? (size_t)c->nz : (size_t)c->nz + 1) * pl;
    TC_CUDA(cudaMemcpyAsync(c->st[c->cur][q], src + q * f, n * 8, cudaMemcpyDeviceToDevice, s));
    TC_CUDA(cudaMemcpyAsync(c->rh[q], src + (3 + q) * f, n * 8, cudaMemcpyDeviceToDevice, s));
  }
  TC_CUDA(cudaMemcpyAsync(c->scal + SC_FORCING, src + 6 * f, 8, cudaMemcpyDeviceToDevice, s));
  c->have_hist = have_hist ? 1 : 0;
  c->state_set = 1;
  return TC_OK;
}

extern "C" int tc_kinetic_energy(tc_ctx* c, double weight, double* acc, void* scratch, void* stream) {
  int rc = adj_check(c, scratch);
  if (rc) return rc;
  if (!acc || !scratch) return fail(TC_ERR_ARG, "null argument");
  if (!c->state_set) return fail(TC_ERR_STATE, "no state");
  cudaStream_t s = ST(stream);
  AdjScratch a = adj_carve(c, scratch);
  double** S = (double**)c->st[c->cur];
  k_ke_partials<<<adj_grid(c), dim3(32, 8), 0, s>>>(S[0], S[1], S[2], c->dzf_d, c->dzc_d, a.partials, c->nx, c->ny,
                                                   c->nz);
  k_ke_finalize<<<1, 256, 0, s>>>(a.partials, (int)adj_nblocks(c), acc,
                                  weight * c->dx * c->dy / (c->Lx * c->Ly * c->Lz));
  TC_LAUNCHED();
  return TC_OK;
}

extern "C" int tc_adjoint_ke_seed(tc_ctx* c, double weight, const double* qu, const double* qv, const double* qw,
                                  double* lu, double* lv, double* lw, void* stream) {
  int rc = adj_check(c, nullptr);
  if (rc) return rc;
  if (!qu || !qv || !qw || !lu || !lv || !lw) return fail(TC_ERR_ARG, "null argument");
  k_ke_seed<<<adj_grid(c), dim3(32, 8), 0, ST(stream)>>>(qu, qv, qw, lu, lv, lw, c->dzf_d, c->dzc_d,
                                                         weight * c->dx * c->dy / (c->Lx * c->Ly * c->Lz), c->nx,
                                                         c->ny, c->nz);
  TC_LAUNCHED();
  return TC_OK;
}

static void adj_rhs_launch(tc_ctx* c, const double* qu, const double* qv, const double* qw, double* const* R,
                           double* lu, double* lv, double* lw, cudaStream_t s) {
  AdjRhsArgs a;
  a.u = qu; a.v = qv; a.w = qw;
  a.Ru = R[0]; a.Rv = R[1]; a.Rw = R[2];
  a.lu = lu; a.lv = lv; a.lw = lw;
  a.idzf = (const double*)c->idzf_t; a.idzc = (const double*)c->idzc_t;
  a.idx = 1.0 / c->dx; a.idy = 1.0 / c->dy;
  a.nu_idx2 = c->nu / (c->dx * c->dx); a.nu_idy2 = c->nu / (c->dy * c->dy);
  a.nx = c->nx; a.ny = c->ny; a.nz = c->nz; a.top_neumann = c->top_neumann; a.rhs_fused = c->rhs_fused;
  k_adj_rhs<<<adj_grid(c), dim3(32, 8), 0, s>>>(a);
}

extern "C" int tc_adjoint_rhs(tc_ctx* c, const double* qu, const double* qv, const double* qw, const double* Ru,
                              const double* Rv, const double* Rw, double* lu, double* lv, double* lw, void* stream) {
  int rc = adj_check(c, nullptr);
  if (rc) return rc;
  if (!qu || !qv || !qw || !Ru || !Rv || !Rw || !lu || !lv || !lw) return fail(TC_ERR_ARG, "null argument");
  double* R[3] = {(double*)Ru, (double*)Rv, (double*)Rw};
  adj_rhs_launch(c, qu, qv, qw, R, lu, lv, lw, ST(stream));
  TC_LAUNCHED();
  return TC_OK;
}

static void adj_cn_launch(tc_ctx* c, double dt, double* lu, double* lv, double* lw, const AdjScratch& a,
                          cudaStream_t s) {
  if (c->adj_tab_dt != dt || c->adj_tab_ptr != a.tab) {  // tables live in the caller's scratch
    k_adj_cn_tables<<<1, 32, 0, s>>>(a.tab, c->dzf_d, c->dzc_d, c->nz, c->nu, dt, c->top_neumann);
    c->adj_tab_dt = dt;
    c->adj_tab_ptr = a.tab;
  }
  k_adj_cn<<<dim3((c->nx * c->ny + 127) / 128, 3), 128, 0, s>>>(lu, lv, lw, a.tab, c->nx, c->ny, c->nz);
}

extern "C" int tc_adjoint_cn(tc_ctx* c, double dt, double* lu, double* lv, double* lw, void* scratch,
                             void* stream) {
  int rc = adj_check(c, scratch);
  if (rc) return rc;
  if (!lu || !lv || !lw || !scratch || !(dt > 0)) return fail(TC_ERR_ARG, "null argument or dt <= 0");
  adj_cn_launch(c, dt, lu, lv, lw, adj_carve(c, scratch), ST(stream));
  TC_LAUNCHED();
  return TC_OK;
}

// lambda <- W P W^-1 (lambda - cb mu grad ub / ...) : see k_adj_scale_in.
static int adj_project_impl(tc_ctx* c, double* lu, double* lv, double* lw, const double* mu, double cb,
                            const AdjScratch& a, cudaStream_t s) {
  k_adj_scale_in<<<adj_grid(c), dim3(32, 8), 0, s>>>(lu, lv, lw, a.A[0], a.A[1], a.A[2], c->dzf_d, c->dzc_d, mu, cb,
                                                    c->nx, c->ny, c->nz);
  int rc = poisson_impl<double>(c, a.A[0], a.A[1], a.A[2], nullptr, c->p, 1.0 / ((double)c->nx * (double)c->ny), s);
  if (rc) return rc;
  k_adj_project_out<<<adj_grid(c), dim3(32, 8), 0, s>>>(a.A[0], a.A[1], a.A[2], c->p, lu, lv, lw, c->dzf_d,
                                                       c->dzc_d, 1.0 / c->dx, 1.0 / c->dy, c->nx, c->ny, c->nz);
  TC_LAUNCHED();
  return TC_OK;
}

extern "C" int tc_adjoint_project(tc_ctx* c, double* lu, double* lv, double* lw, void* scratch, void* stream) {
  int rc = adj_check(c, scratch);
  if (rc) return rc;
  if (!lu || !lv || !lw || !scratch) return fail(TC_ERR_ARG, "null argument");
  return adj_project_impl(c, lu, lv, lw, nullptr, 0.0, adj_carve(c, scratch), ST(stream));
}

extern "C" int tc_adjoint_step(tc_ctx* c, double dt, int first, const double* qu, const double* qv, const double* qw,
                               double* lu, double* lv, double* lw, double* lru, double* lrv, double* lrw,
                               double* lFu, double* lFv, double* lFw, double* mu, void* scratch, void* stream) {
  int rc = adj_check(c, scratch);
  if (rc) return rc;
  if (!qu || !qv || !qw || !lu || !lv || !lw || !lru || !lrv || !lrw || !mu || !scratch || !(dt > 0))
    return fail(TC_ERR_ARG, "null argument or dt <= 0");
  if ((lFu || lFv || lFw) && !(lFu && lFv && lFw)) return fail(TC_ERR_ARG, "lambda_F needs all three or none");
  cudaStream_t s = ST(stream);
  AdjScratch a = adj_carve(c, scratch);
  // bulk velocity / PI forcing, then the projection
  const double cb = 0.1 / dt * c->dx * c->dy / (c->Lx * c->Ly * c->Lz);
  if ((rc = adj_project_impl(c, lu, lv, lw, mu, cb, a, s))) return rc;
  // Crank-Nicolson
  adj_cn_launch(c, dt, lu, lv, lw, a, s);
  // AB2 split, body force, forcing adjoint
  AdjPrepArgs pa;
  pa.l[0] = lu; pa.l[1] = lv; pa.l[2] = lw;
  pa.lr[0] = lru; pa.lr[1] = lrv; pa.lr[2] = lrw;
  for (int q = 0; q < 3; ++q) pa.R[q] = a.R[q];
  pa.F[0] = lFu; pa.F[1] = lFv; pa.F[2] = lFw;
  pa.partials = a.partials;
  pa.c1 = first ? dt : 1.5 * dt;
  pa.c2 = first ? 0.0 : -0.5 * dt;
  pa.nx = c->nx; pa.ny = c->ny; pa.nz = c->nz;
  k_adj_prep<<<adj_grid(c), dim3(32, 8), 0, s>>>(pa);
  k_adj_mu<<<1, 256, 0, s>>>(a.partials, (int)adj_nblocks(c), mu);
  // right-hand side
  adj_rhs_launch(c, qu, qv, qw, a.R, lu, lv, lw, s);
  TC_LAUNCHED();
  return TC_OK;
}

static void drop_graph(tc_ctx* c) {
  if (c->g_valid) {
    cudaGraphExecDestroy(c->gexec);
    c->g_valid = 0;
  }
}

extern "C" int tc_set_ke_accumulator(tc_ctx* c, double* acc, const double* weight_dev, void* scratch) {
  int rc = adj_check(c, scratch);
  if (rc) return rc;
  if (acc && (!weight_dev || !scratch)) return fail(TC_ERR_ARG, "accumulator needs a weight and a scratch");
  c->ke_acc = acc;
  c->ke_w = acc ? weight_dev : nullptr;
  c->ke_part = acc ? adj_carve(c, scratch).partials : nullptr;
  drop_graph(c);
  return TC_OK;
}

extern "C" int tc_set_state_tape(tc_ctx* c, double* tape, int nslots, int* ctr_dev) {
  int rc = adj_check(c, nullptr);
  if (rc) return rc;
  if (tape && (!ctr_dev || nslots < 1)) return fail(TC_ERR_ARG, "tape needs a device counter and nslots >= 1");
  c->tape = tape;
  c->tape_ctr = tape ? ctr_dev : nullptr;
  c->tape_slots = tape ? nslots : 0;
  drop_graph(c);
  return TC_OK;
}

extern "C" int tc_set_cn_chunk(tc_ctx* c, int rows) {
  if (!c) return fail(TC_ERR_ARG, "null ctx");
  if (rows < 0 || rows > 32) return fail(TC_ERR_ARG, "CN chunk length must be 0 .. 32");
  if (rows > 0 && (c->nz + rows - 1) / rows > 16) return fail(TC_ERR_SIZE, "CN chunks of this length exceed 16 per column");
  if (rows != c->cn_L_force) {
    c->cn_L_force = rows;
    c->tab_dt = -1.0;  // the chunk products of the tables follow the length
    drop_graph(c);
  }
  return TC_OK;
}

// ---------------------------------------------------------------------------
// Ensembles: one persistent launch per substep for all members (tc_batch.cuh)
// ---------------------------------------------------------------------------
struct tc_batch {
  int n, precision, dev, nsm;
  std::vector<tc_ctx*> m;
  void* table;               // caller memory: 3 tables of n member records
  size_t rec;                // bytes of one member record
  int cn_L, ctas_per_sm;     // tuned shapes: CN chunk length, CTAs per SM (0: occupancy limit)
  int valid, scheme;         // tables match the members' parity, dt, scheme and shapes
  std::vector<double> dts;
  std::vector<int> cur0;
  int q;                     // steps since the tables were built, mod 2
  int total[BK_COUNT], grid[BK_COUNT];
  int rhs_tma;               // the RHS stages its tiles by tensor copies (kb_rhs_tma)
  std::vector<BatchRhsArgs<float>> rargs_f[3];   // kb_rhs_tma parameters of tables 0, 1, 2, one per member group
  std::vector<BatchRhsArgs<double>> rargs_d[3];
  int cn_y, nmax, fy_tile;   // cn_y: CN chunks of the deepest member
  size_t smem_fy;
  std::vector<int> ccls;     // CN chunk counts of the members, one launch each
  std::vector<int> cmaxnz, cgrid;    // deepest member and CTAs of each CN class
  std::vector<BatchCnArgs<float>> cargs_f[3];   // kb_cn_pk / kb_cn_n parameters of tables 0, 1, 2 per class
  std::vector<BatchCnArgs<double>> cargs_d[3];
  std::vector<int> xcls;     // x-transform lengths N1 of the members, one launch each
  BatchTriArgs targs;        // kb_tri_n parameter
  BatchProjArgs<float> pargs_f[3];   // kb_proj_n parameters of tables 0, 1, 2
  BatchProjArgs<double> pargs_d[3];
  std::vector<BatchXArgs<float>> xargs_f[3];   // kb_fftx_n / kb_ifftx_n parameters per table and class
  std::vector<BatchXArgs<double>> xargs_d[3];
  int graphs_on;
  cudaStream_t cap_stream;
  cudaGraphExec_t gexec;
  int g_valid, g_scheme, g_q;
};

// Whether the ensemble's RHS stages its tiles by tensor copies (kb_rhs_tma):
// every member has its tensor-copy RHS on in the default tile shape, the
// shape of its tensor maps' boxes.  Otherwise kb_rhs runs.
static bool batch_tma_ok(const tc_batch* b) {
  for (const tc_ctx* c : b->m)
    if (!c->rhs_tma_ok || !c->rhs_tma_on || c->rhs_tma_mode != 1) return false;
  return true;
}

static bool batch_grid_ok(const tc_ctx* c) {
  return c->nx % 16 == 0 && c->ny % 16 == 0 && batch_n1_ok(c->nx / 16) && batch_n1_ok(c->ny / 16) &&
         c->ny % XROWS == 0 && c->tri_rden != nullptr;
}

extern "C" int tc_batch_table_bytes(int n, int precision, size_t* bytes) {
  if (!bytes) return fail(TC_ERR_ARG, "null bytes");
  if (n < 1 || n > TC_BATCH_MAX) return fail(TC_ERR_ARG, "ensemble size must be 1 .. 64");
  if (precision != TC_FP64 && precision != TC_MIXED) return fail(TC_ERR_ARG, "bad precision");
  const size_t rec = precision == TC_FP64 ? sizeof(BMember<double>) : sizeof(BMember<float>);
  *bytes = 3 * (size_t)n * rec;
  return TC_OK;
}

static void batch_drop_graph(tc_batch* b) {
  if (b->g_valid) {
    cudaGraphExecDestroy(b->gexec);
    b->g_valid = 0;
  }
}

extern "C" int tc_batch_create(tc_ctx* const* members, int n, void* table, size_t bytes, tc_batch** out) {
  if (!members || !out || !table) return fail(TC_ERR_ARG, "null argument");
  if (n < 1 || n > TC_BATCH_MAX) return fail(TC_ERR_ARG, "ensemble size must be 1 .. 64");
  if (reinterpret_cast<uintptr_t>(table) % 16) return fail(TC_ERR_WORKSPACE, "table must be 16-byte aligned");
  const int prec = members[0] ? members[0]->precision : -1;
  size_t need = 0;
  int rc = tc_batch_table_bytes(n, prec, &need);
  if (rc) return rc;
  if (bytes < need) return fail(TC_ERR_WORKSPACE, "ensemble table too small");
  for (int i = 0; i < n; ++i) {
    const tc_ctx* c = members[i];
    if (!c) return fail(TC_ERR_ARG, "null member");
    if (c->precision != prec) return fail(TC_ERR_ARG, "members must share the precision");
    if (c->dev != members[0]->dev) return fail(TC_ERR_ARG, "members must share the device");
    for (int k = 0; k < i; ++k)
      if (members[k] == c) return fail(TC_ERR_ARG, "a context appears twice in the ensemble");
    if (!batch_grid_ok(c))
      return fail(TC_ERR_SIZE, "ensemble launches need nx, ny in {64, 96, 128, 192, 256}");
  }
  tc_batch* b = new tc_batch();
  b->n = n; b->precision = prec; b->dev = members[0]->dev; b->nsm = members[0]->nsm;
  b->m.assign(members, members + n);
  b->table = table;
  b->rec = prec == TC_FP64 ? sizeof(BMember<double>) : sizeof(BMember<float>);
  int maxnz = 0;
  for (auto* c : b->m) maxnz = std::max(maxnz, c->nz);
  b->cn_L = maxnz <= 256 ? 16 : 32;
  b->ctas_per_sm = 0;
  b->graphs_on = 1;
  *out = b;
  return TC_OK;
}

extern "C" int tc_batch_destroy(tc_batch* b) {
  if (!b) return TC_OK;
  batch_drop_graph(b);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  delete b;
  return TC_OK;
}

extern "C" int tc_batch_set_shape(tc_batch* b, int cn_rows, int ctas_per_sm) {
  if (!b) return fail(TC_ERR_ARG, "null ensemble");
  if (cn_rows != 16 && cn_rows != 32) return fail(TC_ERR_ARG, "CN chunk length must be 16 or 32");
  for (auto* c : b->m)
    if (cn_rows == 16 && c->nz > 256) return fail(TC_ERR_SIZE, "16-row CN chunks need nz <= 256");
  if (ctas_per_sm < -1 || ctas_per_sm > 32) return fail(TC_ERR_ARG, "ctas_per_sm must be -1 .. 32");
  if (cn_rows != b->cn_L || ctas_per_sm != b->ctas_per_sm) {
    b->cn_L = cn_rows;
    b->ctas_per_sm = ctas_per_sm;
    b->valid = 0;
    batch_drop_graph(b);
  }
  return TC_OK;
}

extern "C" int tc_batch_use_graphs(tc_batch* b, int on) {
  if (!b) return fail(TC_ERR_ARG, "null ensemble");
  b->graphs_on = on ? 1 : 0;
  return TC_OK;
}

template <class T> static constexpr int batch_cn_vec(int L) { return (L == 16 && sizeof(T) == 4) ? 2 : 1; }

template <class T>
static BMember<T> batch_record(tc_ctx* c, int cur, double dt, int hist, int scheme, int L) {
  BMember<T> r;
  std::memset(&r, 0, sizeof(r));
  r.g = make_grid<T>(c);
  T** A = (T**)c->st[cur];
  T** Bn = (T**)c->st[cur ^ 1];
  for (int i = 0; i < 3; ++i) { r.A[i] = A[i]; r.B[i] = Bn[i]; r.R[i] = (T*)c->rh[i]; }
  r.forcing = c->scal + SC_FORCING;
  r.dt = (T)dt;
  r.have_hist = hist;
  r.tab = c->tab;
  r.ubase = ubase_of(c);
  r.X = c->X; r.twx = c->twx_d; r.twy = c->twy_d;
  r.scale = 1.0 / (dt * (double)c->nx * (double)c->ny);
  r.rden = c->tri_rden; r.cpt = c->tri_cp;
  r.tb = PoissonTabs{c->k2x, c->k2y, c->cl, c->cr};
  r.p = c->p; r.dzf = c->dzf_d;
  r.ba = BulkArgs{c->partials, c->ticket, c->scal, bulk_scale(c), c->U_bulk, dt, scheme != TC_FE};
  r.n1y = c->ny / 16; r.nxh = c->nxh; r.nrows = c->nxh * c->nz;
  r.rgx = (c->nx + RHS_TX - 1) / RHS_TX;
  r.rgy = (c->ny + rhs_ty<T>() - 1) / rhs_ty<T>();
  r.rgz = (c->nz + 1 + rhs_kb<T>() - 1) / rhs_kb<T>();
  rhs_tma_tiles(c->nx, c->ny, c->nz, BatchRhsTmaShape<T>::KB, &r.tnx, &r.tny, &r.tnz);
  const int V = batch_cn_vec<T>(L);
  r.cgx = (c->nx * c->ny / V + 31) / 32;
  r.xgx = c->ny / XROWS;
  r.xpg = (c->nz + TC_BATCH_XP - 1) / TC_BATCH_XP;
  r.pgx = (c->nx / 2 + 31) / 32; r.pgy = (c->ny + 7) / 8; r.pgz = (c->nz + PROJ_PK - 1) / PROJ_PK;
  return r;
}

template <class T> static void batch_units(const BMember<T>& r, const tc_ctx* c, bool tma, int cnt[BK_COUNT]) {
  cnt[BK_RHS] = tma ? r.tnx * r.tny * r.tnz : r.rgx * r.rgy * r.rgz;
  cnt[BK_CN] = 3 * r.cgx;
  cnt[BK_FX] = r.xgx * r.xpg;
  cnt[BK_FY] = (r.nrows + 1) / 2;
  cnt[BK_TRI] = (2 * c->nxh * c->ny + 63) / 64;
  cnt[BK_IFX] = r.xgx * c->nz;
  cnt[BK_PROJ] = r.pgx * r.pgy * r.pgz;
}

template <class T, class K> static int batch_grid(const tc_batch* b, K kernel, int threads, size_t smem, int total,
                                                  int* grid) {
  int occ = 0;
  TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem));
  if (occ < 1) return fail(TC_ERR_SIZE, "ensemble kernel does not fit on an SM");
  if (b->ctas_per_sm < 0) {  // one CTA per work unit: the hardware scheduler refills the SMs
    *grid = std::max(1, total);
    return TC_OK;
  }
  const int per = b->ctas_per_sm ? std::min(occ, b->ctas_per_sm) : occ;
  *grid = std::max(1, std::min(total, per * b->nsm));
  return TC_OK;
}

// Shared-memory opt-in and persistent grid of every ensemble kernel.
template <class T> static BatchProjArgs<T>* batch_pargs(tc_batch* b) {
  if constexpr (sizeof(T) == 8)
    return b->pargs_d;
  else
    return b->pargs_f;
}
template <class T> static std::vector<BatchCnArgs<T>>* batch_cargs(tc_batch* b) {
  if constexpr (sizeof(T) == 8)
    return b->cargs_d;
  else
    return b->cargs_f;
}
// The CN kernel of chunk length L for blocks of `threads` threads.
template <class T, class F> static void batch_cn_kernel(int L, int threads, F&& f) {
  if (L == 16) {
    if constexpr (sizeof(T) == 4) {
      if (threads <= 256) f(kb_cn_pk<256>); else f(kb_cn_pk<512>);
    } else {
      if (threads <= 256) f(kb_cn_n<T, 16, 256>); else f(kb_cn_n<T, 16, 512>);
    }
  } else {
    if (threads <= 256) f(kb_cn_n<T, 32, 256>); else f(kb_cn_n<T, 32, 512>);
  }
}
template <class T> static size_t batch_cn_smem(int L, int chunks, int maxnz) {
  return (size_t)(9 * maxnz + 2 * chunks * 32 * batch_cn_vec<T>(L)) * 8;
}
// Shared-memory opt-in of each CN class's kernel; one CTA per unit.
template <class T> static int batch_cn_shapes(tc_batch* b) {
  const std::vector<BatchCnArgs<T>>& ca = batch_cargs<T>(b)[0];
  const int nc = (int)b->ccls.size();
  b->cgrid.assign(nc, 1);
  b->grid[BK_CN] = 0;
  int rc = TC_OK;
  for (int c = 0; c < nc && !rc; ++c) {
    const int ch = b->ccls[c];
    const size_t sm = batch_cn_smem<T>(b->cn_L, ch, b->cmaxnz[c]);
    batch_cn_kernel<T>(b->cn_L, 32 * ch, [&](auto k) {
      int occ = 0;
      if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 32 * ch, sm) != cudaSuccess || occ < 1)
        rc = fail(TC_ERR_SIZE, "ensemble CN block does not fit on an SM");
    });
    b->cgrid[c] = std::max(1, ca[c].st[ca[c].n]);
    b->grid[BK_CN] += b->cgrid[c];
  }
  return rc;
}

// Parameters of the CN class launches for the three tables: the members of
// each chunk count (ascending) with their first units (component, column
// block; column blocks fastest).
template <class T> static void batch_cn_args(tc_batch* b, const std::vector<BMember<T>>& tab) {
  const int n = b->n, L = b->cn_L;
  b->ccls.clear();
  for (int i = 0; i < n; ++i) {
    const int ch = (b->m[i]->nz + L - 1) / L;
    if (std::find(b->ccls.begin(), b->ccls.end(), ch) == b->ccls.end()) b->ccls.push_back(ch);
  }
  std::sort(b->ccls.begin(), b->ccls.end());
  b->cmaxnz.assign(b->ccls.size(), 0);
  std::vector<BatchCnArgs<T>>* ca = batch_cargs<T>(b);
  for (int t = 0; t < 3; ++t) {
    ca[t].assign(b->ccls.size(), BatchCnArgs<T>());
    for (size_t c = 0; c < b->ccls.size(); ++c) {
      BatchCnArgs<T>& a = ca[t][c];
      a.n = 0;
      a.st[0] = 0;
      for (int i = 0; i < n; ++i) {
        const tc_ctx* ctx = b->m[i];
        if ((ctx->nz + L - 1) / L != b->ccls[c]) continue;
        const BMember<T>& r = tab[(size_t)t * n + i];
        BCnRec<T>& q = a.r[a.n];
        for (int f = 0; f < 3; ++f) q.B[f] = r.B[f];
        q.tab = r.tab;
        q.ubase = r.ubase;
        q.nx = ctx->nx;
        q.ny = ctx->ny;
        q.nz = ctx->nz;
        q.cgx = r.cgx;
        a.st[a.n + 1] = a.st[a.n] + 3 * r.cgx;
        ++a.n;
        b->cmaxnz[c] = std::max(b->cmaxnz[c], ctx->nz);
      }
    }
  }
}
template <class F> static void batch_n1_host(int n1, F&& f) {
  switch (n1) {
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 12: f(std::integral_constant<int, 12>{}); break;
    default: f(std::integral_constant<int, 16>{}); break;
  }
}
template <class T> static std::vector<BatchXArgs<T>>* batch_xargs(tc_batch* b) {
  if constexpr (sizeof(T) == 8)
    return b->xargs_d;
  else
    return b->xargs_f;
}
template <class T, int NMAX> static int batch_fft_shapes(tc_batch* b) {
  TC_CUDA(cudaFuncSetAttribute(kb_ffty<T, NMAX, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem_fy));
  TC_CUDA(cudaFuncSetAttribute(kb_ffty<T, NMAX, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem_fy));
  int rc = batch_grid<T>(b, kb_ffty<T, NMAX, false>, 128, b->smem_fy, (b->total[BK_FY] + 3) / 4, &b->grid[BK_FY]);
  // x transforms: one launch per length class, one CTA per unit (the grids
  // add up in the info)
  const std::vector<BatchXArgs<T>>& xa = batch_xargs<T>(b)[0];
  const int nc = (int)b->xcls.size();
  b->grid[BK_IFX] = 0;
  b->grid[BK_FX] = 0;
  for (int c = 0; c < nc && !rc; ++c)
    batch_n1_host(b->xcls[c], [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      if (cudaFuncSetAttribute(kb_ifftx_n<T, N1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ifftx_reg_smem<N1>()) != cudaSuccess ||
          cudaFuncSetAttribute(kb_fftx_n<T, N1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)fftx_reg_smem<N1>()) != cudaSuccess) {
        rc = fail(TC_ERR_CUDA, "ensemble x transform attributes");
        return;
      }
      b->grid[BK_IFX] += std::max(1, xa[c].st[xa[c].n]);
      b->grid[BK_FX] += std::max(1, xa[c].stf[xa[c].n]);
    });
  return rc;
}

// Parameters of the x-transform class launches for the three tables: the
// members of each length N1 (ascending) with their first forward and
// inverse units.
template <class T> static void batch_x_args(tc_batch* b, const std::vector<BMember<T>>& tab) {
  const int n = b->n;
  b->xcls.clear();
  for (int i = 0; i < n; ++i) {
    const int n1 = b->m[i]->nx / 16;
    if (std::find(b->xcls.begin(), b->xcls.end(), n1) == b->xcls.end()) b->xcls.push_back(n1);
  }
  std::sort(b->xcls.begin(), b->xcls.end());
  std::vector<BatchXArgs<T>>* xa = batch_xargs<T>(b);
  for (int t = 0; t < 3; ++t) {
    xa[t].assign(b->xcls.size(), BatchXArgs<T>());
    for (size_t c = 0; c < b->xcls.size(); ++c) {
      BatchXArgs<T>& a = xa[t][c];
      a.n = 0;
      a.st[0] = a.stf[0] = 0;
      for (int i = 0; i < n; ++i) {
        const tc_ctx* ctx = b->m[i];
        if (ctx->nx / 16 != b->xcls[c]) continue;
        const BMember<T>& r = tab[(size_t)t * n + i];
        BXRec<T>& q = a.r[a.n];
        q.g = r.g;
        for (int f = 0; f < 3; ++f) q.B[f] = r.B[f];
        q.X = r.X;
        q.twx = r.twx;
        q.p = r.p;
        q.scale = r.scale;
        q.xgx = r.xgx;
        a.st[a.n + 1] = a.st[a.n] + r.xgx * ctx->nz;
        a.stf[a.n + 1] = a.stf[a.n] + r.xgx * r.xpg;
        ++a.n;
      }
    }
  }
}
template <class T> static int batch_shapes(tc_batch* b, int scheme) {
  int rc = batch_cn_shapes<T>(b);
  if (rc) return rc;
  rc = b->nmax == 8 ? batch_fft_shapes<T, 8>(b) : batch_fft_shapes<T, 16>(b);
  if (rc) return rc;
  if (b->rhs_tma) {
    using B = BatchRhsTmaShape<T>;
    const int sm = (int)B::smem();
    auto k0 = kb_rhs_tma<T, false, UPD_AB2>, k1 = kb_rhs_tma<T, true, UPD_AB2>, k2 = kb_rhs_tma<T, true, UPD_FE>;
    TC_CUDA(cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    TC_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    TC_CUDA(cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    rc = batch_grid<T>(b, scheme == TC_IMEX ? k0 : scheme == TC_AB2 ? k1 : k2, RHS_TX * B::S::TY, sm,
                       b->total[BK_RHS], &b->grid[BK_RHS]);
    if (rc) return rc;
  }
  const int rthr = RHS_TX * rhs_ty<T>();
  if (b->rhs_tma)
    rc = TC_OK;
  else if (scheme == TC_IMEX)
    rc = batch_grid<T>(b, kb_rhs<T, false, UPD_AB2>, rthr, 0, b->total[BK_RHS], &b->grid[BK_RHS]);
  else if (scheme == TC_AB2)
    rc = batch_grid<T>(b, kb_rhs<T, true, UPD_AB2>, rthr, 0, b->total[BK_RHS], &b->grid[BK_RHS]);
  else
    rc = batch_grid<T>(b, kb_rhs<T, true, UPD_FE>, rthr, 0, b->total[BK_RHS], &b->grid[BK_RHS]);
  b->grid[BK_TRI] = std::max(1, b->total[BK_TRI]);  // one CTA per unit
  b->grid[BK_PROJ] = std::max(1, b->total[BK_PROJ]);  // one CTA per unit
  return rc;
}

template <class T> static std::vector<BatchRhsArgs<T>>* batch_rargs(tc_batch* b) {
  if constexpr (sizeof(T) == 8)
    return b->rargs_d;
  else
    return b->rargs_f;
}

// Parameters of kb_rhs_tma for the three tables (tab: 3 n member records
// with their first units): per group of TC_BATCH_TMA_GROUP members, each
// member's tensor maps of the parity its table reads (tables 0 and 2: the
// current state, table 1: the other buffer set) and what its tiles read.
template <class T> static void batch_rhs_args(tc_batch* b, const std::vector<BMember<T>>& tab) {
  const int n = b->n, ng = (n + TC_BATCH_TMA_GROUP - 1) / TC_BATCH_TMA_GROUP;
  std::vector<BatchRhsArgs<T>>* ra = batch_rargs<T>(b);
  for (int t = 0; t < 3; ++t) {
    ra[t].assign(ng, BatchRhsArgs<T>());
    for (int i = 0; i < n; ++i) {
      BatchRhsArgs<T>& a = ra[t][i / TC_BATCH_TMA_GROUP];
      const int k = i % TC_BATCH_TMA_GROUP;
      const BMember<T>& r = tab[(size_t)t * n + i];
      const tc_ctx* c = b->m[i];
      const int par = t == 1 ? c->cur ^ 1 : c->cur;
      for (int f = 0; f < 3; ++f) a.map[k][f] = c->tmap[par][f];
      BRhsRec<T>& q = a.r[k];
      q.g = r.g;
      for (int f = 0; f < 3; ++f) { q.A[f] = r.A[f]; q.B[f] = r.B[f]; q.R[f] = r.R[f]; }
      q.forcing = r.forcing;
      q.err = c->err;
      q.dt = r.dt;
      q.have_hist = r.have_hist;
      q.tny = r.tny;
      q.tnz = r.tnz;
      a.st[k] = r.u0[BK_RHS];
      a.st[k + 1] = r.u0[BK_RHS] + r.tnx * r.tny * r.tnz;
      a.nm = k + 1;
    }
  }
}

template <class T> static int batch_build_impl(tc_batch* b, int scheme, const double* dts, cudaStream_t s) {
  const int n = b->n, L = b->cn_L;
  std::vector<BMember<T>> tab(3 * (size_t)n);
  int run[BK_COUNT] = {0, 0, 0, 0, 0, 0, 0};
  int maxnz = 0;
  for (auto* c : b->m) maxnz = std::max(maxnz, c->nz);
  // a member's CN chunks are L rows, like a single-channel step's; one CN
  // launch per chunk count
  const int maxchunks = (maxnz + L - 1) / L;
  b->rhs_tma = batch_tma_ok(b) ? 1 : 0;
  int fyt = 0;
  for (int i = 0; i < n; ++i) {
    tc_ctx* c = b->m[i];
    const int Lr = L;
    if (c->cn_L_force != Lr) {  // the member's CN tables follow its chunk length
      c->cn_L_force = Lr;
      c->tab_dt = -1.0;
      drop_graph(c);
    }
    if (scheme == TC_IMEX && c->tab_dt != dts[i]) {
      launch_cn_tables(c, dts[i], Lr, s);
      TC_LAUNCHED();
      c->tab_dt = dts[i];
    }
    const int hist = scheme == TC_FE ? 0 : c->have_hist;
    tab[i] = batch_record<T>(c, c->cur, dts[i], 1, scheme, L);
    tab[n + i] = batch_record<T>(c, c->cur ^ 1, dts[i], 1, scheme, L);
    tab[2 * n + i] = batch_record<T>(c, c->cur, dts[i], hist, scheme, L);
    int cnt[BK_COUNT];
    batch_units<T>(tab[i], c, b->rhs_tma != 0, cnt);
    for (int k = 0; k < BK_COUNT; ++k) {
      tab[i].u0[k] = tab[n + i].u0[k] = tab[2 * n + i].u0[k] = run[k];
      run[k] += cnt[k];
    }
    for_each_n1(c->ny, [&](auto I) { fyt = std::max(fyt, RowFft<decltype(I)::value>::TILE); });
  }
  for (int k = 0; k < BK_COUNT; ++k) b->total[k] = run[k];
  if (b->rhs_tma) batch_rhs_args<T>(b, tab);
  batch_x_args<T>(b, tab);
  batch_cn_args<T>(b, tab);
  b->targs = BatchTriArgs();
  for (int i = 0; i < n; ++i) {  // the z sweeps read the spectrum: the same for every table
    BTriRec& q = b->targs.r[i];
    q.X = reinterpret_cast<double*>(tab[i].X);
    q.rden = tab[i].rden;
    q.cpt = tab[i].cpt;
    q.tb = tab[i].tb;
    q.nxh = tab[i].nxh;
    q.ny = b->m[i]->ny;
    q.nz = b->m[i]->nz;
    b->targs.st[i] = tab[i].u0[BK_TRI];
  }
  b->targs.st[n] = b->total[BK_TRI];
  b->targs.n = n;
  for (int t = 0; t < 3; ++t) {
    BatchProjArgs<T>& a = batch_pargs<T>(b)[t];
    a = BatchProjArgs<T>();
    for (int i = 0; i < n; ++i) {
      const BMember<T>& r = tab[(size_t)t * n + i];
      BProjRec<T>& q = a.r[i];
      q.g = r.g;
      for (int f = 0; f < 3; ++f) q.B[f] = r.B[f];
      q.p = r.p;
      q.dzf = r.dzf;
      q.ba = r.ba;
      q.pgx = r.pgx;
      q.pgy = r.pgy;
      q.pgz = r.pgz;
      a.st[i] = r.u0[BK_PROJ];
    }
    a.st[n] = b->total[BK_PROJ];
    a.n = n;
  }
  b->cn_y = maxchunks;
  b->fy_tile = fyt;
  b->smem_fy = (size_t)4 * 2 * fyt * sizeof(cpx<double>);
  int n1max = 0;
  for (auto* c : b->m) n1max = std::max(n1max, std::max(c->nx, c->ny) / 16);
  b->nmax = n1max <= 8 ? 8 : 16;
  int rc = batch_shapes<T>(b, scheme);
  if (rc) return rc;
  // pageable copy: returns once the records are staged
  TC_CUDA(cudaMemcpyAsync(b->table, tab.data(), tab.size() * sizeof(BMember<T>), cudaMemcpyHostToDevice, s));
  b->dts.assign(dts, dts + n);
  b->cur0.resize(n);
  for (int i = 0; i < n; ++i) b->cur0[i] = b->m[i]->cur;
  b->q = 0;
  b->scheme = scheme;
  b->valid = 1;
  batch_drop_graph(b);
  return TC_OK;
}

template <class T, int NMAX>
static void batch_poisson(tc_batch* b, const BMember<T>* M, int ti, cudaStream_t s) {
  const int n = b->n;
  const std::vector<BatchXArgs<T>>& xa = batch_xargs<T>(b)[ti];
  for (size_t c = 0; c < xa.size(); ++c)
    batch_n1_host(b->xcls[c], [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      kb_fftx_n<T, N1><<<std::max(1, xa[c].stf[xa[c].n]), 128, fftx_reg_smem<N1>(), s>>>(xa[c]);
    });
  kb_ffty<T, NMAX, false><<<b->grid[BK_FY], 128, b->smem_fy, s>>>(M, n, b->total[BK_FY], b->fy_tile);
  kb_tri_n<<<b->grid[BK_TRI], 64, 0, s>>>(b->targs);
  kb_ffty<T, NMAX, true><<<b->grid[BK_FY], 128, b->smem_fy, s>>>(M, n, b->total[BK_FY], b->fy_tile);
  for (size_t c = 0; c < xa.size(); ++c)
    batch_n1_host(b->xcls[c], [&](auto I) {
      constexpr int N1 = decltype(I)::value;
      kb_ifftx_n<T, N1><<<std::max(1, xa[c].st[xa[c].n]), 128, ifftx_reg_smem<N1>(), s>>>(xa[c]);
    });
}

// One step of every member with table `ti` (0, 1: parity; 2: first step).
template <class T> static int batch_step_impl(tc_batch* b, int scheme, int ti, cudaStream_t s) {
  const BMember<T>* M = reinterpret_cast<const BMember<T>*>(b->table) + (size_t)ti * b->n;
  const int n = b->n;
  const dim3 rb(RHS_TX, rhs_ty<T>());
  if (b->rhs_tma) {
    const dim3 tb(RHS_TX, BatchRhsTmaShape<T>::S::TY);
    const size_t sm = BatchRhsTmaShape<T>::smem();
    for (const BatchRhsArgs<T>& a : batch_rargs<T>(b)[ti]) {  // one launch per member group
      const int gr = std::max(1, std::min(b->grid[BK_RHS], a.st[a.nm] - a.st[0]));
      if (scheme == TC_IMEX)
        kb_rhs_tma<T, false, UPD_AB2><<<gr, tb, sm, s>>>(a);
      else if (scheme == TC_AB2)
        kb_rhs_tma<T, true, UPD_AB2><<<gr, tb, sm, s>>>(a);
      else
        kb_rhs_tma<T, true, UPD_FE><<<gr, tb, sm, s>>>(a);
    }
  } else if (scheme == TC_IMEX)
    kb_rhs<T, false, UPD_AB2><<<b->grid[BK_RHS], rb, 0, s>>>(M, n, b->total[BK_RHS]);
  else if (scheme == TC_AB2)
    kb_rhs<T, true, UPD_AB2><<<b->grid[BK_RHS], rb, 0, s>>>(M, n, b->total[BK_RHS]);
  else
    kb_rhs<T, true, UPD_FE><<<b->grid[BK_RHS], rb, 0, s>>>(M, n, b->total[BK_RHS]);
  if (scheme == TC_IMEX) {  // one launch per chunk count, blocks of (32, chunks)
    const std::vector<BatchCnArgs<T>>& ca = batch_cargs<T>(b)[ti];
    for (size_t c = 0; c < ca.size(); ++c) {
      const int ch = b->ccls[c];
      const size_t sm = batch_cn_smem<T>(b->cn_L, ch, b->cmaxnz[c]);
      batch_cn_kernel<T>(b->cn_L, 32 * ch, [&](auto k) { k<<<b->cgrid[c], dim3(32, ch), sm, s>>>(ca[c]); });
    }
  }
  if (b->nmax == 8)
    batch_poisson<T, 8>(b, M, ti, s);
  else
    batch_poisson<T, 16>(b, M, ti, s);
  kb_proj_n<T><<<b->grid[BK_PROJ], dim3(32, 8), 0, s>>>(batch_pargs<T>(b)[ti]);
  TC_LAUNCHED();
  return TC_OK;
}

static void batch_advance(tc_batch* b, int scheme) {
  for (auto* c : b->m) {
    c->cur ^= 1;
    if (scheme != TC_FE) c->have_hist = 1;
  }
  b->q ^= 1;
}

#define BDISPATCH(b, fn, ...) ((b)->precision == TC_FP64 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

static int batch_build_graph(tc_batch* b, int scheme) {
  batch_drop_graph(b);
  if (!b->cap_stream) TC_CUDA(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
  TC_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
  int rc = TC_OK;
  for (int k = 0; k < 2 && rc == TC_OK; ++k) rc = BDISPATCH(b, batch_step_impl, b, scheme, b->q ^ k, b->cap_stream);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->cap_stream, &graph);
  if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
  if (e != cudaSuccess) return fail(TC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&b->gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(TC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  b->g_valid = 1; b->g_scheme = scheme; b->g_q = b->q;
  return TC_OK;
}

extern "C" int tc_batch_step(tc_batch* b, int scheme, const double* dts, int n_steps, void* stream) {
  if (!b || !dts) return fail(TC_ERR_ARG, "null argument");
  if (scheme != TC_IMEX && scheme != TC_AB2 && scheme != TC_FE) return fail(TC_ERR_ARG, "bad scheme");
  if (n_steps < 0) return fail(TC_ERR_ARG, "n_steps must be >= 0");
  const cudaStream_t s = ST(stream);
  bool rebuild = !b->valid || b->scheme != scheme;
  bool lack = false;
  for (int i = 0; i < b->n; ++i) {
    const tc_ctx* c = b->m[i];
    if (!c->state_set) return fail(TC_ERR_STATE, "member without a state");
    if (!(dts[i] > 0)) return fail(TC_ERR_ARG, "dt must be > 0");
    if (c->body[0] || c->ke_acc || c->tape) return fail(TC_ERR_ARG, "ensemble launches take no adjoint hooks");
    if (c->psp_on) return fail(TC_ERR_ARG, "ensemble launches take no single-precision Poisson members");
    if (b->valid && (b->dts[i] != dts[i] || c->cur != (b->cur0[i] ^ b->q))) rebuild = true;
    if (b->valid && b->rhs_tma != (batch_tma_ok(b) ? 1 : 0)) rebuild = true;
    if (scheme == TC_IMEX && c->tab_dt != dts[i]) rebuild = true;
    lack = lack || (scheme != TC_FE && !c->have_hist);
  }
  if (lack && b->valid && b->q != 0) rebuild = true;
  if (n_steps == 0) return TC_OK;
  if (rebuild) {
    int rc = BDISPATCH(b, batch_build_impl, b, scheme, dts, s);
    if (rc) return rc;
  }
  int k = 0;
  if (lack) {  // first step: members without history take a forward-Euler-style start
    int rc = BDISPATCH(b, batch_step_impl, b, scheme, 2, s);
    if (rc) return rc;
    batch_advance(b, scheme);
    ++k;
  }
  if (b->graphs_on && n_steps - k >= 4) {
    if (!b->g_valid || b->g_scheme != scheme || b->g_q != b->q) {
      int rc = batch_build_graph(b, scheme);
      if (rc) return rc;
    }
    for (; k + 2 <= n_steps; k += 2) {
      TC_CUDA(cudaGraphLaunch(b->gexec, s));
      batch_advance(b, scheme);
      batch_advance(b, scheme);
    }
  }
  for (; k < n_steps; ++k) {
    int rc = BDISPATCH(b, batch_step_impl, b, scheme, b->q, s);
    if (rc) return rc;
    batch_advance(b, scheme);
  }
  return TC_OK;
}

extern "C" int tc_batch_info(tc_batch* b, int* shape, int* units, int* grids) {
  if (!b) return fail(TC_ERR_ARG, "null ensemble");
  if (shape) { shape[0] = b->cn_L; shape[1] = b->ctas_per_sm; shape[2] = b->valid; shape[3] = b->valid ? b->cn_y : 0; }
  for (int k = 0; k < BK_COUNT; ++k) {
    if (units) units[k] = b->valid ? b->total[k] : 0;
    if (grids) grids[k] = b->valid ? b->grid[k] : 0;
  }
  return TC_OK;
}
