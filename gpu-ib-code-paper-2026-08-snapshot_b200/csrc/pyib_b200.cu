// pyib_b200.cu -- B200 (sm_100a) kernels and C ABI for the PyIB per-step hot path.
//
// Layout: dense nested-level boxes (see include/pyib_b200.h).  The CG matvec
// runs as three structured stencil kernels (A: curl+interp, V: viscous block,
// RI: integr+rot) whose rows at level interfaces are replaced inline by
// explicit CSR patch rows.  Step operators (calc_vel, conv_diff, residual
// assembly) run as CSR gathers; they execute a handful of times per step
// against hundreds of CG iterations.  Reductions are deterministic: fixed grid
// sizes, per-block partial sums, and a fixed-order final sum by the last block.
//
// Build with --fmad=false so every scalar expression rounds like the NumPy
// reference (no contracted multiply-adds).
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pyib_b200.h"

#define PYIB_VERSION "pyib_b200 0.1.0 sm_100a"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;      // fixed grid of the flat vector kernels (148 SMs x 8)
constexpr int kPartStride = 65536;       // partial-sum slots per reduction value (>= any grid)
constexpr int kSlots = 16;               // reduction values per block
// structured stencil tiles: 32 x 8 threads in (x, y), each marching KZ planes in z
constexpr int TX = 32, TY = 8;
constexpr int kTargetBlocks = 148 * 16;   // z-chunk depth is chosen to give at least this many tiles
// fused matvec blocks: 32 x 16 threads over a column tile with a 2-column halo below and
// 1 above, owning 29 x 13 node columns; at most kMaxKzF node planes per block
constexpr int FX = 32, FY = 16, FOX = FX - 3, FOY = FY - 3;
constexpr int kMaxKzF = 32;

struct LevelMeta {
  int n[3];
  int hole_lo[3];
  int hole_hi[3];      // exclusive
  int has_hole;
  double h;
  long long cbase;
  long long fbase[3];
  long long ebase[3];
  long long ecount[3];
  double prec_reg;     // preconditioner value of the level's regular edges
  int plane_base;      // first per-plane partial-sum slot of this level (kernel RI)
  int zbA;             // first z-block of this level in the cell-tile grids
  int zbR;             // first z-block of this level in the node-tile grid
  int zbF;             // first z-block of this level in the fused-matvec grid
  int fplane_base;     // first per-plane partial-sum slot of this level (fused matvec)
};

struct Meta {
  int nl;
  LevelMeta lv[PYIB_MAX_LEVELS];
  long long nc, nf, ne;
  int kz;              // z planes marched by one cell tile (kernels A and V)
  int kzR;             // z planes marched by one node tile (kernel RI)
  int gxA, gyA, gzA;   // cell-tile grid (kernel A; kernel V uses gxV and the same y, z)
  int gxV;             // x tiles of kernel V (two cells per thread: 64 cells a tile)
  int gxR, gyR, gzR;   // node-tile grid (kernel RI)
  int nplanes;         // per-plane partial sums of kernel RI (independent of the z-chunk depth)
  int ri_up;           // 1: kernel RI also marches the upper-face nodes (i = nx, j = ny, k = nz);
                       // 0: every upper-face edge is an exact (patch) row or masked
  int av;              // 1: kernels A and V run fused (k_mvAV); 0: as two kernels
  int kzF;             // node planes marched by one block of the fused matvec
  int gxF, gyF, gzF;   // fused-matvec grid
  int nplanesF;        // per-plane partial sums of the fused matvec
};

struct CGState {
  double eta, eta_new, pw, alpha, beta, thresh, l2_0, xnorm;
  double true_eta, true_l2, tol1, tol2;
  double rou, kfac;              // V block: rou*v - kfac*(Vd v)
  double thresh_in;              // inner (float32) stop threshold of the mixed solver
  int m, done, iters, check, cg_max, alpd, stop, pad1;
  unsigned int counter;
  unsigned int counter2;
};

struct Table {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct pyib_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  pyib_layout lay{};
  Meta meta{};
  pyib_params prm{};
  bool have_params = false;
  Table tab[PYIB_T_COUNT];
  long long nA = 0, nV = 0, nR = 0;   // patch rows
  long long n_inlet = 0, n_bf = 0, n_cand = 0, n_fidx = 0;
  // fields
  double *s = nullptr, *s_old = nullptr, *U = nullptr, *vc = nullptr, *res_c0 = nullptr,
         *res_c = nullptr, *res_e = nullptr, *F = nullptr, *fE = nullptr, *conv = nullptr,
         *diff = nullptr;
  double *work_e = nullptr, *work_e2 = nullptr, *work_c3 = nullptr, *work_f = nullptr;
  // CG vectors
  double *x = nullptr, *r = nullptr, *p = nullptr, *w = nullptr, *vcm = nullptr, *vq = nullptr,
         *prev = nullptr;
  float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *w32 = nullptr, *vcm32 = nullptr,
        *vq32 = nullptr, *prec32 = nullptr;
  float *pa_val32 = nullptr, *pv_val32 = nullptr, *pr_val32 = nullptr;
  double *diag1 = nullptr, *diag2 = nullptr;   // diag(R I P C) and diag(R I Vd' P C)
  double diag_for_kfac = -1.0, diag_for_rou = -1.0;
  bool diag_ready = false;
  cudaGraphExec_t mix_graph = nullptr;
  int mix_graph_check = 0;
  long long mix_graph_kernels = 0;   // kernel nodes in mix_graph
  // reduction / state
  double* partials = nullptr;
  CGState* st = nullptr;
  CGState* st_host = nullptr;     // pinned
  // IB
  int M = 0;
  double *mk = nullptr, *mvel = nullptr, *ds = nullptr, *fL = nullptr, *lag = nullptr,
         *dL = nullptr, *ibw = nullptr;
  int *ibcell = nullptr, *ibbase = nullptr;
  double* ibjac = nullptr;        // 9 per marker: d u_L / d x_marker (pyib_ib_interp_dx)
  void* ws = nullptr;             // grow-only workspace of the offline graph calls
  size_t ws_bytes = 0;
  void* ws_tmp = nullptr;         // grow-only CUB temporary storage of those calls
  size_t ws_tmp_bytes = 0;
  int imp_iters = 0;              // CG iterations of the last implicit IB solve
  int *sort_keys_in = nullptr, *sort_keys_out = nullptr, *sort_vals_in = nullptr,
      *sort_vals_out = nullptr;
  void* sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;
  double pos_ref[3] = {0, 0, 0};
  double dx = 0.0;
  int ib_n[3] = {0, 0, 0};
  bool stencil_valid = false;
  int* dev_err = nullptr;          // kernel-side error word
  // graphs
  cudaGraphExec_t cg_graph = nullptr;
  int cg_graph_check = 0;
  long long cg_graph_kernels = 0;    // kernel nodes in cg_graph
  int cg_graph_alpd = -1;
  // fused single-pass matvec of the float64 CG (k_mvF)
  bool use_fused = false;        // PYIB_FUSED_MATVEC=1 selects the single-pass matvec in the CG
  int av_pin = -1;               // PYIB_MATVEC_AV: -1 tuned, 0 kernels A and V apart, 1 fused
  bool fused_ready = false;
  bool flags_ready = false;      // f_* cell flags and the f_list of the fused kernels
  bool tunedF = false;
  unsigned int *f_irrA = nullptr, *f_irrV = nullptr, *f_needR = nullptr;
  unsigned char* f_flags = nullptr;   // per cell: exact vc / exact vq / store vq
  int* f_list = nullptr;         // regular cells whose template vc an exact V row reads
  long long n_list = 0;
  // timing
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, tev0 = nullptr, tev1 = nullptr;
  double cg_seconds = 0.0;
  long long cg_iters = 0;
  long long launches = 0;        // kernels launched by this context
  bool tuned = false;            // matvec tile depths chosen by timing
  Meta meta32{};                 // the float32 matvec's copy of meta, with its own tile depths
  bool tuned32 = false;
  double tune_ms = 0.0;          // best matvec time seen by the tuner
};

namespace {

int set_err(pyib_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return set_err(ctx, PYIB_E_CUDA, "%s failed: %s (%s:%d)", #call,                \
                     cudaGetErrorString(e_), __FILE__, __LINE__);                      \
  } while (0)

#define CKL()                                                                          \
  do {                                                                                 \
    ++ctx->launches;                                                                   \
    cudaError_t e_ = cudaGetLastError();                                               \
    if (e_ != cudaSuccess)                                                             \
      return set_err(ctx, PYIB_E_CUDA, "kernel launch failed: %s (%s:%d)",             \
                     cudaGetErrorString(e_), __FILE__, __LINE__);                      \
  } while (0)

#define RET(call)                   \
  do {                              \
    int rc_ = (call);               \
    if (rc_ != PYIB_OK) return rc_; \
  } while (0)

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > kMaxBlocks) b = kMaxBlocks;
  return (int)b;
}

// one thread per patch row, every row at once: fixed for a given row count
int patch_grid(long long rows) {
  long long b = (rows + kThreads - 1) / kThreads;
  return (int)(b < 1 ? 1 : b);
}

// ---------------------------------------------------------------------------
// deterministic block reduction
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh /*[NV*32]*/) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double t = v[q];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[q * 32 + wid] = t;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x * blockDim.y * blockDim.z) >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double t = lane < nw ? sh[q * 32 + lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      v[q] = t;
    }
  }
  __syncthreads();
}

// Sum of partials[base + b] for b in [0, n) by one block: each thread adds its
// stride-blockDim subsequence into four accumulators (L2 loads, independent, so they
// pipeline), then the block tree.  Fixed order for a given n and block size.
__device__ __forceinline__ double strided_sum(const double* partials, int n) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int q = tid;
  for (; q + 3 * nt < n; q += 4 * nt) {
    a0 += __ldcg(partials + q);
    a1 += __ldcg(partials + q + nt);
    a2 += __ldcg(partials + q + 2 * nt);
    a3 += __ldcg(partials + q + 3 * nt);
  }
  for (; q < n; q += nt) a0 += __ldcg(partials + q);
  return (a0 + a1) + (a2 + a3);
}

// Block coordinates of a kernel body: the launch's own (blockIdx, gridDim), or, in a
// batched launch over several cases, the block's coordinates within its case's grid.
struct Grid3 {
  int bx, by, bz, gx, gy, gz;
};
struct Grid1 {
  int b, nb;   // block and block count of a one-dimensional grid
};
__device__ __forceinline__ Grid3 own_grid3() {
  return Grid3{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, (int)gridDim.x, (int)gridDim.y, (int)gridDim.z};
}
__device__ __forceinline__ Grid1 own_grid1() { return Grid1{(int)blockIdx.x, (int)gridDim.x}; }

// Writes this block's partials; returns true in the block that finishes last (of the
// nb blocks counted on counter), whose thread 0 then holds the totals in v (summed
// in block order).
template <int NV>
__device__ bool grid_sum_at(double (&v)[NV], double* partials, unsigned int* counter, unsigned int bid,
                            unsigned int nb) {
  __shared__ double sh[NV * 32];
  __shared__ bool last;
  block_sum<NV>(v, sh);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[q * kPartStride + bid] = v[q];
    __threadfence();
    unsigned int t = atomicAdd(counter, 1u);
    last = (t == nb - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = strided_sum(partials + (size_t)q * kPartStride, (int)nb);
  (void)nthr;
  block_sum<NV>(acc, sh);
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = acc[q];
    *counter = 0u;
  }
  return tid == 0;
}

template <int NV>
__device__ bool grid_sum(double (&v)[NV], double* partials, unsigned int* counter) {
  return grid_sum_at<NV>(v, partials, counter, blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
                         gridDim.x * gridDim.y * gridDim.z);
}

// ---------------------------------------------------------------------------
// layout decoding
// ---------------------------------------------------------------------------


__device__ __forceinline__ bool bit_set(const unsigned int* bits, long long i) {
  return (bits[i >> 5] >> (i & 31)) & 1u;
}

__device__ __forceinline__ int level_of_zblock(const Meta& m, int bz, bool node_grid) {
  int L = 0;
  while (L + 1 < m.nl && bz >= (node_grid ? m.lv[L + 1].zbR : m.lv[L + 1].zbA)) ++L;
  return L;
}

// Grids of the structured kernels for z-chunk depths kzA (cells) and kzR (nodes).
void set_grids(Meta& m, int kzA, int kzR) {
  m.kz = kzA;
  m.kzR = kzR;
  int zA = 0, zR = 0, gxA = 1, gyA = 1, gxR = 1, gyR = 1, gxV = 1;
  for (int L = 0; L < m.nl; ++L) {
    LevelMeta& l = m.lv[L];
    l.zbA = zA;
    l.zbR = zR;
    zA += (l.n[2] + kzA - 1) / kzA;
    zR += (l.n[2] + m.ri_up + kzR - 1) / kzR;
    gxA = std::max(gxA, (l.n[0] + TX - 1) / TX);
    gxV = std::max(gxV, (l.n[0] + 2 * TX - 1) / (2 * TX));
    gyA = std::max(gyA, (l.n[1] + TY - 1) / TY);
    gxR = std::max(gxR, (l.n[0] + m.ri_up + TX - 1) / TX);
    gyR = std::max(gyR, (l.n[1] + m.ri_up + TY - 1) / TY);
  }
  m.gxA = gxA; m.gyA = gyA; m.gzA = zA; m.gxV = gxV;
  m.gxR = gxR; m.gyR = gyR; m.gzR = zR;
  int pb = 0;
  for (int L = 0; L < m.nl; ++L) {
    m.lv[L].plane_base = pb;
    pb += gxR * gyR * (m.lv[L].n[2] + m.ri_up);
  }
  m.nplanes = pb;
}

// Grid of the fused matvec for z-chunk depth kzF (node planes per block).
void set_grids_fused(Meta& m, int kzF) {
  m.kzF = kzF;
  int z = 0, gx = 1, gy = 1;
  for (int L = 0; L < m.nl; ++L) {
    LevelMeta& l = m.lv[L];
    l.zbF = z;
    z += (l.n[2] + m.ri_up + kzF - 1) / kzF;
    gx = std::max(gx, (l.n[0] + m.ri_up + FOX - 1) / FOX);
    gy = std::max(gy, (l.n[1] + m.ri_up + FOY - 1) / FOY);
  }
  m.gxF = gx; m.gyF = gy; m.gzF = z;
  int pb = 0;
  for (int L = 0; L < m.nl; ++L) {
    m.lv[L].fplane_base = pb;
    pb += gx * gy * (m.lv[L].n[2] + m.ri_up);
  }
  m.nplanesF = pb;
}

// ---------------------------------------------------------------------------
// matvec kernel A: vc = P C p.  Thread (i,j) of a 32x8 tile marches KZ cell planes;
// the two x- and y-edge values of the upper plane are carried to the next plane.
// Irregular cells (hole neighbours, interface cells) take their exact CSR rows.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void mvA_tile(const Meta& m, Grid3 g, const T* __restrict__ p, T* __restrict__ vc) {
  const int L = level_of_zblock(m, g.bz, false);
  const LevelMeta& l = m.lv[L];
  const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
  const int i = g.bx * TX + threadIdx.x, j = g.by * TY + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const int k0 = (g.bz - l.zbA) * m.kz;
  const int k1 = min(k0 + m.kz, nz);
  const long long nc = m.nc;
  const T* ex = p + l.ebase[0];
  const T* ey = p + l.ebase[1];
  const T* ez = p + l.ebase[2];
  const int sxk = (ny + 1) * nx, syk = ny * (nx + 1), szk = (ny + 1) * (nx + 1);
  int ox = (k0 * (ny + 1) + j) * nx + i;
  int oy = (k0 * ny + j) * (nx + 1) + i;
  int oz = (k0 * (ny + 1) + j) * (nx + 1) + i;
  T ex00 = ex[ox], ex10 = ex[ox + nx];
  T ey00 = ey[oy], ey10 = ey[oy + 1];
  const T s = (T)(1.0 / (2.0 * l.h * l.h));
  const bool col_hole = l.has_hole && i >= l.hole_lo[0] && i < l.hole_hi[0] && j >= l.hole_lo[1] &&
                        j < l.hole_hi[1];
  long long c = l.cbase + ((long long)k0 * ny + j) * nx + i;
  const long long cstep = (long long)nx * ny;
  for (int k = k0; k < k1; ++k, c += cstep, ox += sxk, oy += syk, oz += szk) {
    const T ex01 = ex[ox + sxk], ex11 = ex[ox + sxk + nx];
    const T ey01 = ey[oy + syk], ey11 = ey[oy + syk + 1];
    if (!(col_hole && k >= l.hole_lo[2] && k < l.hole_hi[2])) {
      // template for every cell; rows of irregular cells are overwritten by k_patchA
      const T ez00 = ez[oz], ez10 = ez[oz + 1], ez01 = ez[oz + nx + 1], ez11 = ez[oz + nx + 2];
      const T ux0 = ey00 + ez01 - ey01 - ez00;
      const T ux1 = ey10 + ez11 - ey11 - ez10;
      const T uy0 = ez00 + ex01 - ez10 - ex00;
      const T uy1 = ez01 + ex11 - ez11 - ex10;
      const T uz0 = ex00 + ey10 - ex10 - ey00;
      const T uz1 = ex01 + ey11 - ex11 - ey01;
      vc[c] = (ux0 + ux1) * s;
      vc[nc + c] = (uy0 + uy1) * s;
      vc[2 * nc + c] = (uz0 + uz1) * s;
    }
    ex00 = ex01; ex10 = ex11; ey00 = ey01; ey10 = ey11;
  }
}

template <typename T>
__global__ void __launch_bounds__(TX * TY) k_mvA(Meta m, const T* __restrict__ p, T* __restrict__ vc,
                                                  const unsigned int* __restrict__ pbits,
                                                  const int* __restrict__ prow,
                                                  const long long* __restrict__ pptr,
                                                  const int* __restrict__ pcol,
                                                  const T* __restrict__ pval, long long nA,
                                                  const CGState* __restrict__ st) {
  if (st && st->done) return;
  mvA_tile<T>(m, own_grid3(), p, vc);
}

// ---------------------------------------------------------------------------
// matvec kernel V: vq = rou v - kfac * Vd v per component (7-point template with a
// zero ghost at the domain boundary).  Each thread owns two x-consecutive cells
// (a tile is 64 x 8 cells), so the pair shares its x-neighbour loads; the
// z-neighbours are carried in registers.  Hole cells are skipped; rows of
// irregular cells are overwritten by k_patchV.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void mvV_tile(const Meta& m, Grid3 g, const T* __restrict__ v, T* __restrict__ vq,
                                         const CGState* __restrict__ st) {
  const int L = level_of_zblock(m, g.bz, false);
  const LevelMeta& l = m.lv[L];
  const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
  const int i = g.bx * (2 * TX) + 2 * threadIdx.x, j = g.by * TY + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const bool hasB = i + 1 < nx;                   // the second cell (i+1, j)
  const int k0 = (g.bz - l.zbA) * m.kz;
  const int k1 = min(k0 + m.kz, nz);
  const long long nc = m.nc;
  const T rou = (T)st->rou, kf = (T)st->kfac;
  const T inv_h2 = (T)(1.0 / (l.h * l.h));
  const int cs = nx * ny;
  const bool row_hole = l.has_hole && j >= l.hole_lo[1] && j < l.hole_hi[1];
  const bool holeA = row_hole && i >= l.hole_lo[0] && i < l.hole_hi[0];
  const bool holeB = row_hole && i + 1 >= l.hole_lo[0] && i + 1 < l.hole_hi[0];
  const bool xm = i > 0, xpB = i + 2 < nx, ym = j > 0, yp = j + 1 < ny;
  const long long off = l.cbase + (long long)k0 * cs + (long long)j * nx + i;
  const T* src = v + off;
  T* dst = vq + off;
  T am[3], a0[3], bm[3], b0[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const T* sd = src + d * nc;
    a0[d] = sd[0];
    b0[d] = hasB ? sd[1] : (T)0;
    am[d] = k0 > 0 ? sd[-cs] : (T)0;
    bm[d] = (k0 > 0 && hasB) ? sd[1 - cs] : (T)0;
  }
  for (int k = k0; k < k1; ++k) {
    const bool zp = k + 1 < nz, zm = k > 0;
    const bool zhole = k >= l.hole_lo[2] && k < l.hole_hi[2];
    const bool doA = !(holeA && zhole), doB = hasB && !(holeB && zhole);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T* sd = src + d * nc;
      const T ap = zp ? sd[cs] : (T)0;
      const T bp = (zp && hasB) ? sd[cs + 1] : (T)0;
      if (doA) {
        const T x0 = a0[d];
        T acc = 0;
        acc += hasB ? b0[d] - x0 : -2 * x0;
        acc += xm ? sd[-1] - x0 : -2 * x0;
        acc += yp ? sd[nx] - x0 : -2 * x0;
        acc += ym ? sd[-nx] - x0 : -2 * x0;
        acc += zp ? ap - x0 : -2 * x0;
        acc += zm ? am[d] - x0 : -2 * x0;
        dst[d * nc] = rou * x0 - kf * (acc * inv_h2);
      }
      if (doB) {
        const T x0 = b0[d];
        T acc = 0;
        acc += xpB ? sd[2] - x0 : -2 * x0;
        acc += a0[d] - x0;
        acc += yp ? sd[nx + 1] - x0 : -2 * x0;
        acc += ym ? sd[1 - nx] - x0 : -2 * x0;
        acc += zp ? bp - x0 : -2 * x0;
        acc += zm ? bm[d] - x0 : -2 * x0;
        dst[d * nc + 1] = rou * x0 - kf * (acc * inv_h2);
      }
      am[d] = a0[d]; a0[d] = ap; bm[d] = b0[d]; b0[d] = bp;
    }
    src += cs;
    dst += cs;
  }
}

template <typename T>
__global__ void __launch_bounds__(TX * TY) k_mvV(Meta m, const T* __restrict__ v, T* __restrict__ vq,
                                                  const CGState* __restrict__ st) {
  if (st->done) return;
  mvV_tile<T>(m, own_grid3(), v, vq, st);
}

// ---------------------------------------------------------------------------
// matvec kernel AV: vq = V P C p in one pass (kernels A and V fused), so the cell
// intermediate vc stays on chip.  Thread (tx,ty) of a 32x8 cell tile marches KZ cell
// planes in z and computes vc one plane ahead of the viscous row that needs it.  The
// x/y neighbours of the 7-point template come from a two-plane shared-memory buffer
// holding vc of the tile and of its one-cell ring; the z neighbours stay in registers.
// The ring columns are marched by warps 0-2 (warp 0 the row below the tile, warp 1 the
// row above, warp 2 the columns left (lanes 0-7) and right (lanes 16-23)); every
// column carries its upper x- and y-edge values to the next plane, as kernel A does.
// Cells with exact vc rows (kFlagExactVc) take vc from vcm, where k_patchA wrote it
// before this kernel; the template vc of the cells an exact V row reads (kFlagStoreVc)
// is stored to vcm for k_patchV, which runs after this kernel and overwrites the vq
// of irregular cells.  Every row is the expression of k_mvA and k_mvV term for term,
// so vq is bit-identical to the two-kernel path.
// ---------------------------------------------------------------------------
// per-cell flags of the fused matvec kernels: exact vc row (k_patchA), exact vq row
// (k_patchV), vq read by an exact w row (k_mvF stores it), template vc read by an
// exact vq row (k_mvAV stores it)
constexpr unsigned char kFlagExactVc = 1, kFlagExactVq = 2, kFlagStoreVq = 4, kFlagStoreVc = 8;

template <typename T>
struct AVCol {
  int ox, oy, oz;          // x-, y-, z-edge offsets of the column's cell on the next plane
  T ex0, ex1, ey0, ey1;    // x-edges (i,j), (i,j+1) and y-edges (i,j), (i+1,j) of that plane
};

template <typename T>
__device__ __forceinline__ void av_col_start(AVCol<T>& c, const T* ex, const T* ey, int nx, int ny, int i, int j,
                                             int k) {
  c.ox = (k * (ny + 1) + j) * nx + i;
  c.oy = (k * ny + j) * (nx + 1) + i;
  c.oz = (k * (ny + 1) + j) * (nx + 1) + i;
  c.ex0 = ex[c.ox];
  c.ex1 = ex[c.ox + nx];
  c.ey0 = ey[c.oy];
  c.ey1 = ey[c.oy + 1];
}

// template vc of the column's cell on its next plane when tmpl (else v is left as is),
// then the column moves up one plane
template <typename T>
__device__ __forceinline__ void av_col_step(AVCol<T>& c, const T* ex, const T* ey, const T* ez, int nx, int sxk,
                                            int syk, int szk, T s, bool tmpl, T (&v)[3]) {
  const T ex01 = ex[c.ox + sxk], ex11 = ex[c.ox + sxk + nx];
  const T ey01 = ey[c.oy + syk], ey11 = ey[c.oy + syk + 1];
  // the z-edges are loaded whatever the cell's flag (they exist for every cell of the
  // level's box), so these loads are not held up by the flag load
  const T ez00 = ez[c.oz], ez10 = ez[c.oz + 1], ez01 = ez[c.oz + nx + 1], ez11 = ez[c.oz + nx + 2];
  if (tmpl) {
    const T ux0 = c.ey0 + ez01 - ey01 - ez00;
    const T ux1 = c.ey1 + ez11 - ey11 - ez10;
    const T uy0 = ez00 + ex01 - ez10 - c.ex0;
    const T uy1 = ez01 + ex11 - ez11 - c.ex1;
    const T uz0 = c.ex0 + c.ey1 - c.ex1 - c.ey0;
    const T uz1 = ex01 + ey11 - ex11 - ey01;
    v[0] = (ux0 + ux1) * s;
    v[1] = (uy0 + uy1) * s;
    v[2] = (uz0 + uz1) * s;
  }
  c.ex0 = ex01;
  c.ex1 = ex11;
  c.ey0 = ey01;
  c.ey1 = ey11;
  c.ox += sxk;
  c.oy += syk;
  c.oz += szk;
}

// vc of cell (i,j,k) of the column: exact (vcm), zero in the hole, else the template
template <typename T>
__device__ __forceinline__ void av_col_vc(AVCol<T>& c, const LevelMeta& l, const T* ex, const T* ey, const T* ez,
                                          const T* vcm, const unsigned char* __restrict__ flags, long long nc,
                                          int sxk, int syk, int szk, T s, bool col_hole, int i, int j, int k,
                                          unsigned char& f, T (&v)[3]) {
  const int nx = l.n[0], ny = l.n[1];
  const long long cell = l.cbase + ((long long)k * ny + j) * nx + i;
  f = flags[cell];
  const bool hole = col_hole && k >= l.hole_lo[2] && k < l.hole_hi[2];
  const bool exact = (f & kFlagExactVc) != 0;
  av_col_step<T>(c, ex, ey, ez, nx, sxk, syk, szk, s, !hole && !exact, v);
  if (exact) {
    v[0] = vcm[cell];
    v[1] = vcm[nc + cell];
    v[2] = vcm[2 * nc + cell];
  } else if (hole) {
    v[0] = v[1] = v[2] = (T)0;
  }
}

template <typename T>
__global__ void __launch_bounds__(TX * TY, sizeof(T) == 8 ? 3 : 4) k_mvAV(Meta m, const T* __restrict__ p, T* vcm, T* __restrict__ vq,
                                                   const unsigned char* __restrict__ flags,
                                                   const CGState* __restrict__ st) {
  static_assert(TX == 32 && TY == 8, "the ring assignment below assumes 32 x 8 tiles");
  if (st->done) return;
  __shared__ T sv[2][3][TY + 2][TX + 2];
  const int L = level_of_zblock(m, blockIdx.z, false);
  const LevelMeta& l = m.lv[L];
  const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  if (i0 >= nx || j0 >= ny) return;   // the whole block lies outside this level
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = i < nx && j < ny;
  const int k0 = (blockIdx.z - l.zbA) * m.kz;
  const int k1 = min(k0 + m.kz, nz);
  const long long nc = m.nc;
  const T* ex = p + l.ebase[0];
  const T* ey = p + l.ebase[1];
  const T* ez = p + l.ebase[2];
  const int sxk = (ny + 1) * nx, syk = ny * (nx + 1), szk = (ny + 1) * (nx + 1);
  const T s = (T)(1.0 / (2.0 * l.h * l.h));
  const T rou = (T)st->rou, kf = (T)st->kfac;
  const T inv_h2 = (T)(1.0 / (l.h * l.h));
  auto in_hole_col = [&](int a, int b) {
    return l.has_hole && a >= l.hole_lo[0] && a < l.hole_hi[0] && b >= l.hole_lo[1] && b < l.hole_hi[1];
  };
  // ring column of this thread (shared-memory slot sx, sy), if any
  int hi = -1, hj = -1, sx = 0, sy = 0;
  if (ty == 0) { hi = i; hj = j0 - 1; sx = tx + 1; sy = 0; }
  else if (ty == 1) { hi = i; hj = j0 + TY; sx = tx + 1; sy = TY + 1; }
  else if (ty == 2 && tx < TY) { hi = i0 - 1; hj = j0 + tx; sx = 0; sy = tx + 1; }
  else if (ty == 2 && tx >= 16 && tx < 16 + TY) { hi = i0 + TX; hj = j0 + tx - 16; sx = TX + 1; sy = tx - 15; }
  const bool ring = hi >= 0 && hi < nx && hj >= 0 && hj < ny;
  const bool own_hole = in_hole_col(i, j), ring_hole = ring && in_hole_col(hi, hj);
  const int kstart = k0 > 0 ? k0 - 1 : 0;
  AVCol<T> oc, rc;
  if (own) av_col_start<T>(oc, ex, ey, nx, ny, i, j, kstart);
  if (ring) av_col_start<T>(rc, ex, ey, nx, ny, hi, hj, kstart);
  T vm[3] = {0, 0, 0}, v0[3] = {0, 0, 0}, vp[3] = {0, 0, 0}, hv[3] = {0, 0, 0};
  unsigned char f = 0;
  if (k0 > 0) {
    // plane k0-1: the own column's z-lower neighbour; the ring column only moves up
    if (own) av_col_vc<T>(oc, l, ex, ey, ez, vcm, flags, nc, sxk, syk, szk, s, own_hole, i, j, k0 - 1, f, vm);
    if (ring) av_col_step<T>(rc, ex, ey, ez, nx, sxk, syk, szk, s, false, hv);
  }
  if (own) {
    av_col_vc<T>(oc, l, ex, ey, ez, vcm, flags, nc, sxk, syk, szk, s, own_hole, i, j, k0, f, v0);
    if (f & kFlagStoreVc) {
      const long long cell = l.cbase + ((long long)k0 * ny + j) * nx + i;
      vcm[cell] = v0[0];
      vcm[nc + cell] = v0[1];
      vcm[2 * nc + cell] = v0[2];
    }
  }
  if (ring) av_col_vc<T>(rc, l, ex, ey, ez, vcm, flags, nc, sxk, syk, szk, s, ring_hole, hi, hj, k0, f, hv);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    sv[0][d][ty + 1][tx + 1] = v0[d];
    if (ring) sv[0][d][sy][sx] = hv[d];
  }
  __syncthreads();
  const bool xp = i + 1 < nx, xm = i > 0, yp = j + 1 < ny, ym = j > 0;
  for (int k = k0; k < k1; ++k) {
    const int b = (k - k0) & 1;
    const bool next = k + 1 < k1;   // plane k+1 is this block's: the ring goes to shared memory
    if (k + 1 < nz) {
      if (own) {
        av_col_vc<T>(oc, l, ex, ey, ez, vcm, flags, nc, sxk, syk, szk, s, own_hole, i, j, k + 1, f, vp);
        if (next && (f & kFlagStoreVc)) {
          const long long cell = l.cbase + ((long long)(k + 1) * ny + j) * nx + i;
          vcm[cell] = vp[0];
          vcm[nc + cell] = vp[1];
          vcm[2 * nc + cell] = vp[2];
        }
      }
      if (next && ring)
        av_col_vc<T>(rc, l, ex, ey, ez, vcm, flags, nc, sxk, syk, szk, s, ring_hole, hi, hj, k + 1, f, hv);
      if (next) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          sv[b ^ 1][d][ty + 1][tx + 1] = vp[d];
          if (ring) sv[b ^ 1][d][sy][sx] = hv[d];
        }
      }
    }
    if (own && !(own_hole && k >= l.hole_lo[2] && k < l.hole_hi[2])) {
      const bool zp = k + 1 < nz, zm = k > 0;
      T* dst = vq + l.cbase + ((long long)k * ny + j) * nx + i;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const T x0 = v0[d];
        T acc = 0;
        acc += xp ? sv[b][d][ty + 1][tx + 2] - x0 : -2 * x0;
        acc += xm ? sv[b][d][ty + 1][tx] - x0 : -2 * x0;
        acc += yp ? sv[b][d][ty + 2][tx + 1] - x0 : -2 * x0;
        acc += ym ? sv[b][d][ty][tx + 1] - x0 : -2 * x0;
        acc += zp ? vp[d] - x0 : -2 * x0;
        acc += zm ? vm[d] - x0 : -2 * x0;
        dst[d * nc] = rou * x0 - kf * (acc * inv_h2);
      }
    }
    if (next) __syncthreads();
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      vm[d] = v0[d];
      v0[d] = vp[d];
    }
  }
}

// ---------------------------------------------------------------------------
// matvec kernel RI: w = R I vq, fused with the dot p.w (alpha = eta / p.w is set by
// k_patchRI).  Thread (i,j) of a 32x8 node tile marches kz node planes.  The face values
//   F_x(i,j,k) = (h/2)(vq_x(i-1,j,k) + vq_x(i,j,k)),  F_y likewise in y,
//   F_z(i,j,k) = (h/2)(vq_z(i,j,k-1) + vq_z(i,j,k))
// of the node and of its -x and -y neighbours come straight from (L1-cached)
// loads; the z-lower values are carried from the previous plane.
//   w_x(i,j,k) = F_z(i,j,k) - F_z(i,j-1,k) + F_y(i,j,k-1) - F_y(i,j,k)
//   w_y(i,j,k) = F_x(i,j,k) - F_x(i,j,k-1) + F_z(i-1,j,k) - F_z(i,j,k)
//   w_z(i,j,k) = F_y(i,j,k) - F_y(i-1,j,k) + F_x(i,j-1,k) - F_x(i,j,k)
// The nodes on a level's upper faces (i = nx, j = ny, k = nz) carry only interface
// and boundary edges.  When all of those are exact (patch) rows or masked -- every
// closed-cavity layout -- the kernel marches only nodes i < nx, j < ny, k < nz
// (ri_up = 0), so the node tiles are whole 32 x 8 tiles of the cell grid; otherwise
// (ri_up = 1) it marches all nx+1 x ny+1 x nz+1 nodes.
// ---------------------------------------------------------------------------
template <typename T>
struct RICarry {
  T vz00, vzm0, vz0m;   // vq_z of cells (i,j), (i-1,j), (i,j-1) on the previous plane
  T fy, fx;             // F_y(i,j), F_x(i,j) on the previous plane
};

// carried values of node (i,j) entering plane k0
template <typename T>
__device__ __forceinline__ void ri_start(const LevelMeta& l, int i, int j, int k0, const T* vx, const T* vy,
                                         const T* vz, T hh, RICarry<T>& c) {
  const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
  const bool c00 = i < nx && j < ny, cm0 = i > 0 && i <= nx && j < ny, c0m = i < nx && j > 0 && j <= ny;
  c.vz00 = c.vzm0 = c.vz0m = c.fy = c.fx = (T)0;
  if (k0 > 0) {
    const int ob = (k0 - 1) * (nx * ny) + j * nx + i;
    c.vz00 = c00 ? vz[ob] : (T)0;
    c.vzm0 = cm0 ? vz[ob - 1] : (T)0;
    c.vz0m = c0m ? vz[ob - nx] : (T)0;
    if (k0 - 1 < nz) {
      if (i < nx) c.fy = hh * ((c0m ? vy[ob - nx] : (T)0) + (c00 ? vy[ob] : (T)0));
      if (j < ny) c.fx = hh * ((cm0 ? vx[ob - 1] : (T)0) + (c00 ? vx[ob] : (T)0));
    }
  }
}

// the three edges of node (i,j) on plane k; returns their share of p.w (template edges)
template <typename T>
__device__ __forceinline__ double ri_plane(const LevelMeta& l, int i, int j, int k, const T* vx, const T* vy,
                                           const T* vz, T hh, T* __restrict__ w, const T* __restrict__ p,
                                           const unsigned int* __restrict__ pbits, int do_dot, RICarry<T>& c) {
  const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
  const bool c00 = i < nx && j < ny, cm0 = i > 0 && i <= nx && j < ny, c0m = i < nx && j > 0 && j <= ny,
             cmm = i > 0 && j > 0 && i <= nx && j <= ny;
  const bool zin = k < nz;
  const int ob = k * (nx * ny) + j * nx + i;
  const long long ex_e = l.ebase[0] + (long long)k * ((ny + 1) * nx) + j * nx + i;
  const long long ey_e = l.ebase[1] + (long long)k * (ny * (nx + 1)) + j * (nx + 1) + i;
  const long long ez_e = l.ebase[2] + (long long)k * ((ny + 1) * (nx + 1)) + j * (nx + 1) + i;
  // loads that do not depend on the stencil: bitmask words and the dot's p values
  const unsigned int bwx = (pbits && i < nx) ? pbits[ex_e >> 5] : 0u;
  const unsigned int bwy = (pbits && j < ny) ? pbits[ey_e >> 5] : 0u;
  const unsigned int bwz = (pbits && zin) ? pbits[ez_e >> 5] : 0u;
  const T px = (do_dot && i < nx) ? p[ex_e] : (T)0;
  const T py = (do_dot && j < ny) ? p[ey_e] : (T)0;
  const T pz = (do_dot && zin) ? p[ez_e] : (T)0;
  const T vz00 = (zin && c00) ? vz[ob] : (T)0;
  const T vzm0 = (zin && cm0) ? vz[ob - 1] : (T)0;
  const T vz0m = (zin && c0m) ? vz[ob - nx] : (T)0;
  T fx = 0, fy = 0, fx_jm = 0, fy_im = 0;
  if (zin) {
    const T vx00 = c00 ? vx[ob] : (T)0, vxm0 = cm0 ? vx[ob - 1] : (T)0;
    const T vy00 = c00 ? vy[ob] : (T)0, vy0m = c0m ? vy[ob - nx] : (T)0;
    if (j < ny) fx = hh * (vxm0 + vx00);                                                     // F_x(i,j)
    if (i < nx) fy = hh * (vy0m + vy00);                                                     // F_y(i,j)
    if (j > 0) fx_jm = hh * ((cmm ? vx[ob - nx - 1] : (T)0) + (c0m ? vx[ob - nx] : (T)0));   // F_x(i,j-1)
    if (i > 0) fy_im = hh * ((cmm ? vy[ob - nx - 1] : (T)0) + (cm0 ? vy[ob - 1] : (T)0));    // F_y(i-1,j)
  }
  const T fz = (i < nx && j < ny) ? hh * (c.vz00 + vz00) : (T)0;                             // F_z(i,j)
  const T fz_im = (i > 0 && j < ny) ? hh * (c.vzm0 + vzm0) : (T)0;                           // F_z(i-1,j)
  const T fz_jm = (i < nx && j > 0) ? hh * (c.vz0m + vz0m) : (T)0;                           // F_z(i,j-1)
  // template for every edge; irregular edges are overwritten by k_patchRI, which also
  // adds their share of the dot product
  double dot = 0.0;
  if (i < nx) {
    const T val = fz - fz_jm + c.fy - fy;
    w[ex_e] = val;
    if (!((bwx >> (ex_e & 31)) & 1u)) dot += (double)px * (double)val;
  }
  if (j < ny) {
    const T val = fx - c.fx + fz_im - fz;
    w[ey_e] = val;
    if (!((bwy >> (ey_e & 31)) & 1u)) dot += (double)py * (double)val;
  }
  if (zin) {
    const T val = fy - fy_im + fx_jm - fx;
    w[ez_e] = val;
    if (!((bwz >> (ez_e & 31)) & 1u)) dot += (double)pz * (double)val;
  }
  c.vz00 = vz00; c.vzm0 = vzm0; c.vz0m = vz0m;
  c.fx = fx; c.fy = fy;
  return dot;
}

template <typename T>
__device__ __forceinline__ void mvRI_tile(const Meta& m, Grid3 g, const T* __restrict__ vq, T* __restrict__ w,
                                          const T* __restrict__ p, const unsigned int* __restrict__ pbits,
                                          double* partials, int do_dot) {
  static_assert(TY == 8, "the per-plane combine below assumes 8 warps per block");
  __shared__ double swarp[16][TY];
  const int L = level_of_zblock(m, g.bz, true);
  const LevelMeta& l = m.lv[L];
  const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
  const int i = g.bx * TX + threadIdx.x, j = g.by * TY + threadIdx.y;
  const int k0 = (g.bz - l.zbR) * m.kzR;
  const int k1 = min(k0 + m.kzR, nz + m.ri_up);
  const long long nc = m.nc;
  const T* vx = vq + l.cbase;
  const T* vy = vq + nc + l.cbase;
  const T* vz = vq + 2 * nc + l.cbase;
  const T hh = (T)(0.5 * l.h);
  const bool act = i < nx + m.ri_up && j < ny + m.ri_up;
  RICarry<T> c;
  if (act) ri_start<T>(l, i, j, k0, vx, vy, vz, hh, c);
  for (int k = k0; k < k1; ++k) {
    const double dot = act ? ri_plane<T>(l, i, j, k, vx, vy, vz, hh, w, p, pbits, do_dot, c) : 0.0;
    if (do_dot) {
      // warp sum of this plane, kept per (plane, warp) until the end of the block
      double t = dot;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (threadIdx.x == 0) swarp[k - k0][threadIdx.y] = t;
    }
  }
  if (!do_dot) return;
  __syncthreads();
  // one partial per (level, tile, plane), combined in a fixed order: the sum does not
  // depend on the z-chunk depth the autotuner picked
  const int tid = threadIdx.x + TX * threadIdx.y;
  if (tid < k1 - k0) {
    const double* q = swarp[tid];
    const double v = ((q[0] + q[4]) + (q[2] + q[6])) + ((q[1] + q[5]) + (q[3] + q[7]));
    partials[l.plane_base + ((k0 + tid) * m.gyR + g.by) * m.gxR + g.bx] = v;
  }
}

template <typename T>
__global__ void __launch_bounds__(TX * TY) k_mvRI(Meta m, const T* __restrict__ vq, T* __restrict__ w,
                                                   const T* __restrict__ p,
                                                   const unsigned int* __restrict__ pbits, double* partials,
                                                   CGState* st, int do_dot) {
  if (st->done) return;
  mvRI_tile<T>(m, own_grid3(), vq, w, p, pbits, partials, do_dot);
}

// ---------------------------------------------------------------------------
// Patch kernels: exact CSR rows of the entities the templates cannot reproduce
// (interfaces between levels, hole surfaces, collapsed edges).  One thread per
// row and a grid that covers every row at once: rows are short (about 8
// entries), so the cost is one dependent gather chain per row, overlapped
// across all rows.
// ---------------------------------------------------------------------------
// The row is read in chunks of 8 entries: the chunk's columns and values are
// loaded first, then its gathers, then the products are added in entry order,
// so the sum is the sequential one and only the loads overlap.
template <typename T>
__device__ __forceinline__ T csr_row(const long long* __restrict__ ptr, const int* __restrict__ col,
                                     const T* __restrict__ val, const T* __restrict__ src, long long r) {
  const long long q0 = ptr[r], q1 = ptr[r + 1];
  T acc = 0;
  for (long long q = q0; q < q1; q += 8) {
    int cc[8];
    T vv[8], xs[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const bool ok = q + u < q1;
      cc[u] = ok ? col[q + u] : 0;
      vv[u] = ok ? val[q + u] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) xs[u] = (q + u < q1) ? src[cc[u]] : (T)0;
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (q + u < q1) acc += vv[u] * xs[u];
  }
  return acc;
}

// vc rows: row q = d*nA + r holds component d of cell ids[r]
template <typename T>
__device__ __forceinline__ void patchA_rows(Grid1 g, long long nA, const int* __restrict__ ids,
                                            const long long* __restrict__ ptr, const int* __restrict__ col,
                                            const T* __restrict__ val, const T* __restrict__ p, T* vc,
                                            long long nc) {
  const long long q = g.b * (long long)blockDim.x + threadIdx.x;
  if (q >= 3 * nA) return;
  vc[(q / nA) * nc + ids[q % nA]] = csr_row<T>(ptr, col, val, p, q);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_patchA(long long nA, const int* __restrict__ ids,
                                                     const long long* __restrict__ ptr,
                                                     const int* __restrict__ col, const T* __restrict__ val,
                                                     const T* __restrict__ p, T* vc, long long nc,
                                                     const CGState* __restrict__ st) {
  if (st->done) return;
  patchA_rows<T>(own_grid1(), nA, ids, ptr, col, val, p, vc, nc);
}

// vq rows: the same Vd row for the three components of cell ids[r], one thread per row
// (the row's columns and values are loaded once for the three gathers)
template <typename T>
__device__ __forceinline__ void patchV_rows(Grid1 g, long long nV, const int* __restrict__ ids,
                                            const long long* __restrict__ ptr, const int* __restrict__ col,
                                            const T* __restrict__ val, const T* __restrict__ v, T* vq, long long nc,
                                            const CGState* __restrict__ st) {
  const long long r = g.b * (long long)blockDim.x + threadIdx.x;
  if (r >= nV) return;
  const int c = ids[r];
  const long long q0 = ptr[r], q1 = ptr[r + 1];
  T a0 = 0, a1 = 0, a2 = 0;
  // chunks of 4 entries, loads first, products added in entry order (as csr_row)
  for (long long q = q0; q < q1; q += 4) {
    int cc[4];
    T vv[4], x0[4], x1[4], x2[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool ok = q + u < q1;
      cc[u] = ok ? col[q + u] : 0;
      vv[u] = ok ? val[q + u] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool ok = q + u < q1;
      x0[u] = ok ? v[cc[u]] : (T)0;
      x1[u] = ok ? v[nc + cc[u]] : (T)0;
      x2[u] = ok ? v[2 * nc + cc[u]] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (q + u < q1) {
        a0 += vv[u] * x0[u];
        a1 += vv[u] * x1[u];
        a2 += vv[u] * x2[u];
      }
  }
  const T rou = (T)st->rou, kf = (T)st->kfac;
  vq[c] = rou * v[c] - kf * a0;
  vq[nc + c] = rou * v[nc + c] - kf * a1;
  vq[2 * nc + c] = rou * v[2 * nc + c] - kf * a2;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_patchV(long long nV, const int* __restrict__ ids,
                                                     const long long* __restrict__ ptr,
                                                     const int* __restrict__ col, const T* __restrict__ val,
                                                     const T* __restrict__ v, T* vq, long long nc,
                                                     const CGState* __restrict__ st) {
  if (st->done) return;
  patchV_rows<T>(own_grid1(), nV, ids, ptr, col, val, v, vq, nc, st);
}

// w rows (columns index the component-major vq), plus their share of p.w; the
// per-plane partials of k_mvRI and the rows' shares are summed in a fixed order
// (independent of the z-chunk depth) and the last block sets alpha = eta / p.w.
template <typename T>
__device__ __forceinline__ void patchRI_rows(Grid1 g, long long nR, const int* __restrict__ ids,
                                             const long long* __restrict__ ptr, const int* __restrict__ col,
                                             const T* __restrict__ val, const T* __restrict__ vq, T* w,
                                             const T* __restrict__ p, double* partials, int nplanes, CGState* st,
                                             int do_dot) {
  const long long r = g.b * (long long)blockDim.x + threadIdx.x;
  double dot[1] = {0.0};
  if (r < nR) {
    const int e = ids[r];
    const T acc = csr_row<T>(ptr, col, val, vq, r);
    w[e] = acc;
    if (do_dot) dot[0] = (double)p[e] * (double)acc;
  }
  if (!do_dot) return;
  __shared__ double sh[2 * 32];
  __shared__ bool last;
  // Two-stage fixed-order sum: each block adds a fixed slice of k_mvRI's per-plane
  // partials to its own rows' share, and the last block sums one value per block.
  const int per = (nplanes + g.nb - 1) / g.nb;
  const int q0 = min(nplanes, g.b * per), q1 = min(nplanes, q0 + per);
  double v2[2] = {dot[0], 0.0};
  for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) v2[1] += partials[q];
  block_sum<2>(v2, sh);
  if (threadIdx.x == 0) {
    partials[nplanes + g.b] = v2[0] + v2[1];
    __threadfence();
    last = atomicAdd(&st->counter, 1u) == (unsigned int)g.nb - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc[1] = {strided_sum(partials + nplanes, g.nb)};
  block_sum<1>(acc, sh);
  if (threadIdx.x == 0) {
    st->pw = acc[0];
    st->alpha = st->eta / (acc[0] != 0.0 ? acc[0] : INFINITY);
    st->counter = 0u;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_patchRI(long long nR, const int* __restrict__ ids,
                                                      const long long* __restrict__ ptr,
                                                      const int* __restrict__ col, const T* __restrict__ val,
                                                      const T* __restrict__ vq, T* w, const T* __restrict__ p,
                                                      double* partials, int nplanes, CGState* st, int do_dot) {
  if (st->done) return;
  patchRI_rows<T>(own_grid1(), nR, ids, ptr, col, val, vq, w, p, partials, nplanes, st, do_dot);
}

// ---------------------------------------------------------------------------
// Fused single-pass float64 matvec: w = R I V P C p and the dot p.w in one kernel.
//
// Block of FX x FY = 32 x 16 threads; thread (tx, ty) owns the cell/node column
// (I, J) = (FOX*bx - 2 + tx, FOY*by - 2 + ty) of one level and marches z.  At node
// plane k the block computes, in registers and shared memory only:
//   vc(k+1) = P C p on every column            (12 edge loads per cell, L1)
//   vq(k)   = V vc on columns 1 <= tx, ty < 31/15   (x neighbours by shuffle,
//             y neighbours from shared memory, z neighbours in registers)
//   w(k)    = R I vq on the owned nodes 2 <= tx < 31, 2 <= ty < 15  (29 x 13)
// so the cell intermediates vc and vq never reach DRAM: the kernel reads p once
// (each tile stages its planes of p, halo included, into shared memory with
// cp.async two planes ahead of use) and writes w once.  The arithmetic of every template row
// is the expression of k_mvA / k_mvV / ri_plane, term for term, so w is bit-identical
// to the three-kernel path.  Rows the templates cannot reproduce keep their exact
// CSR rows: k_patchA (vc of irregular cells) and k_vc_list (template vc of the
// cells those rows read) and k_patchV (vq of irregular cells) run before, into the
// same vcm / vq buffers, and this kernel takes vc / vq of a flagged cell from there;
// it also stores the template vq of the cells that the exact w rows of k_patchRI
// read, and k_patchRI runs after it as in the three-kernel path.
// ---------------------------------------------------------------------------

struct FusedTabs {
  const unsigned int* irrA;    // cell bits: exact vc in vcm (k_patchA)
  const unsigned int* irrV;    // cell bits: exact vq in vq (k_patchV)
  const unsigned int* needR;   // cell bits: k_patchRI reads this cell's vq
  const unsigned int* pbits;   // edge bits: exact (patch) w rows, outside the template dot
  const unsigned char* flags;  // the three cell bits as one byte per cell (k_cell_flags)
};

__device__ __forceinline__ int level_of_zblock_fused(const Meta& m, int bz) {
  int L = 0;
  while (L + 1 < m.nl && bz >= m.lv[L + 1].zbF) ++L;
  return L;
}

// template vc of cell (i, j, k) of level l (the arithmetic of k_mvA)
__device__ __forceinline__ void vc_template(const LevelMeta& l, const double* __restrict__ p, int i, int j, int k,
                                            double& vx, double& vy, double& vz) {
  const int nx = l.n[0], ny = l.n[1];
  const double* ex = p + l.ebase[0];
  const double* ey = p + l.ebase[1];
  const double* ez = p + l.ebase[2];
  const int sxk = (ny + 1) * nx, syk = ny * (nx + 1);
  const int ox = (k * (ny + 1) + j) * nx + i;
  const int oy = (k * ny + j) * (nx + 1) + i;
  const int oz = (k * (ny + 1) + j) * (nx + 1) + i;
  const double ex00 = ex[ox], ex10 = ex[ox + nx], ex01 = ex[ox + sxk], ex11 = ex[ox + sxk + nx];
  const double ey00 = ey[oy], ey10 = ey[oy + 1], ey01 = ey[oy + syk], ey11 = ey[oy + syk + 1];
  const double ez00 = ez[oz], ez10 = ez[oz + 1], ez01 = ez[oz + nx + 1], ez11 = ez[oz + nx + 2];
  const double s = 1.0 / (2.0 * l.h * l.h);
  const double ux0 = ey00 + ez01 - ey01 - ez00;
  const double ux1 = ey10 + ez11 - ey11 - ez10;
  const double uy0 = ez00 + ex01 - ez10 - ex00;
  const double uy1 = ez01 + ex11 - ez11 - ex10;
  const double uz0 = ex00 + ey10 - ex10 - ey00;
  const double uz1 = ex01 + ey11 - ex11 - ey01;
  vx = (ux0 + ux1) * s;
  vy = (uy0 + uy1) * s;
  vz = (uz0 + uz1) * s;
}

// Shared-memory staging of p: one node plane of the tile holds the x-edges of
// 32 x 17 node columns, the y-edges of 33 x 16 and the z-edges of 33 x 17 (the
// 12 edges of every cell of the 32 x 16 column block).  Planes are copied with
// cp.async two planes ahead of their use into a ring of kPRing planes, so the
// loads of a plane are in flight while the block computes the previous ones.
// Each block tabulates once, in shared memory, the in-plane source offset of
// every staged element (or -1 outside the level box), so a plane's copies cost a
// table read, one multiply-add and the copy instruction each.
constexpr int FPX = FX + 1, FPY = FY + 1;
constexpr int kPEx = FX * FPY;                  // 544 x-edges a plane
constexpr int kPEy = FPX * FY;                  // 528 y-edges
constexpr int kPEz = FPX * FPY;                 // 561 z-edges
constexpr int kPPlane = kPEx + kPEy + kPEz;     // 1633 doubles
constexpr int kPRing = 5;
constexpr int kPIter = (kPPlane + FX * FY - 1) / (FX * FY);   // staged elements per thread and plane
constexpr size_t kFusedSmemBytes =
    (size_t)(kPRing * kPPlane + 2 * 3 * FY * FX + 3 * FY * FX + kMaxKzF * FY) * sizeof(double) +
    (size_t)kPPlane * sizeof(int);

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = ok ? 8 : 0;   // 0 source bytes: the 8 destination bytes are zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ int ring_slot(int kp) { return ((kp % kPRing) + kPRing) % kPRing; }

// In-plane source offsets of the staged elements of the tile whose column (0, 0)
// is (x0, y0): offset of the edge within its array's plane, -1 outside the box.
__device__ __forceinline__ void tabulate_p_offsets(const LevelMeta& l, int* s_poff, int x0, int y0, int tid) {
  const int nx = l.n[0], ny = l.n[1];
  for (int q = tid; q < kPPlane; q += FX * FY) {
    int off = -1;
    if (q < kPEx) {
      const int yy = q / FX, xx = q - yy * FX, I = x0 + xx, J = y0 + yy;
      if (I >= 0 && I < nx && J >= 0 && J <= ny) off = J * nx + I;
    } else if (q < kPEx + kPEy) {
      const int r = q - kPEx, yy = r / FPX, xx = r - yy * FPX, I = x0 + xx, J = y0 + yy;
      if (I >= 0 && I <= nx && J >= 0 && J < ny) off = J * (nx + 1) + I;
    } else {
      const int r = q - kPEx - kPEy, yy = r / FPX, xx = r - yy * FPX, I = x0 + xx, J = y0 + yy;
      if (I >= 0 && I <= nx && J >= 0 && J <= ny) off = J * (nx + 1) + I;
    }
    s_poff[q] = off;
  }
}

// Issue the copies of node plane kp into ring slot `slot`; elements outside the
// level box (offset -1) or its planes are zero-filled.
__device__ __forceinline__ void load_p_plane(const LevelMeta& l, const double* __restrict__ p, double* slot,
                                             const int* s_poff, int kp, int tid) {
  const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
  const bool pxy = kp >= 0 && kp <= nz, pz = kp >= 0 && kp < nz;
  const double* bx = p + l.ebase[0] + (pxy ? kp * ((ny + 1) * nx) : 0);
  const double* by = p + l.ebase[1] + (pxy ? kp * (ny * (nx + 1)) : 0);
  const double* bz = p + l.ebase[2] + (pz ? kp * ((ny + 1) * (nx + 1)) : 0);
#pragma unroll
  for (int u = 0; u < kPIter; ++u) {
    const int q = tid + u * FX * FY;
    if (q < kPPlane) {
      const int off = s_poff[q];
      const double* base = q < kPEx ? bx : (q < kPEx + kPEy ? by : bz);
      const bool ok = off >= 0 && (q < kPEx + kPEy ? pxy : pz);
      cp_async8(slot + q, ok ? base + off : p, ok);
    }
  }
}

// template vc of the cell of column (tx, ty) on plane kc from the staged planes kc and
// kc + 1 (the arithmetic of k_mvA); s = 1 / (2 h^2)
__device__ __forceinline__ void vc_staged(const double* pa, const double* pb, int tx, int ty, double s,
                                          double& vx, double& vy, double& vz) {
  const double ex00 = pa[ty * FX + tx], ex10 = pa[(ty + 1) * FX + tx];
  const double ex01 = pb[ty * FX + tx], ex11 = pb[(ty + 1) * FX + tx];
  const double* ya = pa + kPEx;
  const double* yb = pb + kPEx;
  const double ey00 = ya[ty * FPX + tx], ey10 = ya[ty * FPX + tx + 1];
  const double ey01 = yb[ty * FPX + tx], ey11 = yb[ty * FPX + tx + 1];
  const double* za = pa + kPEx + kPEy;
  const double ez00 = za[ty * FPX + tx], ez10 = za[ty * FPX + tx + 1];
  const double ez01 = za[(ty + 1) * FPX + tx], ez11 = za[(ty + 1) * FPX + tx + 1];
  const double ux0 = ey00 + ez01 - ey01 - ez00;
  const double ux1 = ey10 + ez11 - ey11 - ez10;
  const double uy0 = ez00 + ex01 - ez10 - ex00;
  const double uy1 = ez01 + ex11 - ez11 - ex10;
  const double uz0 = ex00 + ey10 - ex10 - ey00;
  const double uz1 = ex01 + ey11 - ex11 - ey01;
  vx = (ux0 + ux1) * s;
  vy = (uy0 + uy1) * s;
  vz = (uz0 + uz1) * s;
}

__global__ void __launch_bounds__(FX * FY, 2) k_mvF(Meta m, const double* __restrict__ p, double* __restrict__ w,
                                                   const double* __restrict__ vcm, double* vq, FusedTabs tb,
                                                   double* partials, const CGState* __restrict__ st, int do_dot) {
  if (st->done) return;
  extern __shared__ double fsm[];
  double* ring = fsm;                                                   // [kPRing][kPPlane]
  double (*s_vc)[3][FY][FX] = reinterpret_cast<double (*)[3][FY][FX]>(fsm + kPRing * kPPlane);
  double (*s_vq)[FY][FX] = reinterpret_cast<double (*)[FY][FX]>(fsm + kPRing * kPPlane + 2 * 3 * FY * FX);
  double (*s_dot)[FY] = reinterpret_cast<double (*)[FY]>(fsm + kPRing * kPPlane + 2 * 3 * FY * FX + 3 * FY * FX);
  int* s_poff = reinterpret_cast<int*>(fsm + kPRing * kPPlane + 2 * 3 * FY * FX + 3 * FY * FX + kMaxKzF * FY);
  const int L = level_of_zblock_fused(m, blockIdx.z);
  const LevelMeta& l = m.lv[L];
  const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + FX * ty;
  const int x0 = blockIdx.x * FOX - 2, y0 = blockIdx.y * FOY - 2;
  const int I = x0 + tx, J = y0 + ty;
  const int k0 = (blockIdx.z - l.zbF) * m.kzF;
  const int k1 = min(k0 + m.kzF, nz + m.ri_up);
  const int nc = (int)m.nc;
  const bool col = I >= 0 && I < nx && J >= 0 && J < ny;
  const bool col_hole = l.has_hole && I >= l.hole_lo[0] && I < l.hole_hi[0] && J >= l.hole_lo[1] &&
                        J < l.hole_hi[1];
  const int hz0 = col_hole ? l.hole_lo[2] : 0, hz1 = col_hole ? l.hole_hi[2] : 0;
  const bool do_vq = tx >= 1 && tx < FX - 1 && ty >= 1 && ty < FY - 1;
  const bool own = tx >= 2 && tx < FX - 1 && ty >= 2 && ty < FY - 1;      // owned node (I >= 0, J >= 0)
  const bool do_w = own && I < nx + m.ri_up && J < ny + m.ri_up;
  const double rou = st->rou, kf = st->kfac;
  const double inv_h2 = 1.0 / (l.h * l.h);
  const double s_a = 1.0 / (2.0 * l.h * l.h);
  const double hh = 0.5 * l.h;
  const int cplane = nx * ny;
  const int ccol = (int)l.cbase + J * nx + I;     // cell id of (I, J, 0)
  const int exs = (ny + 1) * nx, eys = ny * (nx + 1), ezs = (ny + 1) * (nx + 1);
  const int ex0 = (int)l.ebase[0] + J * nx + I, ey0 = (int)l.ebase[1] + J * (nx + 1) + I,
            ez0 = (int)l.ebase[2] + J * (nx + 1) + I;   // edges of node (I, J, 0)

  auto cell_in = [&](int kc) { return col && kc >= 0 && kc < nz && !(kc >= hz0 && kc < hz1); };
  auto flag_of = [&](int kc) -> unsigned int { return cell_in(kc) ? tb.flags[ccol + kc * cplane] : 0u; };
  auto inc = [](int s) { return s + 1 == kPRing ? 0 : s + 1; };

  tabulate_p_offsets(l, s_poff, x0, y0, tid);
  __syncthreads();
  // node planes k0-2 .. k0+1 (one group) and k0+2 (a second group)
  for (int kp = k0 - 2; kp <= k0 + 1; ++kp) load_p_plane(l, p, ring + ring_slot(kp) * kPPlane, s_poff, kp, tid);
  cp_async_commit();
  load_p_plane(l, p, ring + ring_slot(k0 + 2) * kPPlane, s_poff, k0 + 2, tid);
  cp_async_commit();
  unsigned int fm = flag_of(k0 - 2), f0 = flag_of(k0 - 1), f1 = flag_of(k0);
  cp_async_wait<1>();
  __syncthreads();
  double am[3] = {0.0, 0.0, 0.0}, a0[3] = {0.0, 0.0, 0.0}, ap[3];
  {
    // vc on planes k0-2 and k0-1
    const int sa = ring_slot(k0 - 2), sb = inc(sa), sc = inc(sb);
    if (cell_in(k0 - 2)) {
      const int c = ccol + (k0 - 2) * cplane;
      if (fm & kFlagExactVc) {
        am[0] = vcm[c]; am[1] = vcm[nc + c]; am[2] = vcm[2 * nc + c];
      } else {
        vc_staged(ring + sa * kPPlane, ring + sb * kPPlane, tx, ty, s_a, am[0], am[1], am[2]);
      }
    }
    if (cell_in(k0 - 1)) {
      const int c = ccol + (k0 - 1) * cplane;
      if (f0 & kFlagExactVc) {
        a0[0] = vcm[c]; a0[1] = vcm[nc + c]; a0[2] = vcm[2 * nc + c];
      } else {
        vc_staged(ring + sb * kPPlane, ring + sc * kPPlane, tx, ty, s_a, a0[0], a0[1], a0[2]);
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) s_vc[(k0 - 1) & 1][d][ty][tx] = a0[d];
  __syncthreads();
  // carried values of node (I, J) from plane k-1 (ri_plane's RICarry)
  double c_vz00 = 0.0, c_vzm0 = 0.0, c_vz0m = 0.0, c_fx = 0.0, c_fy = 0.0;
  int sk = ring_slot(k0 - 1);          // ring slot of node plane k
  for (int k = k0 - 1; k < k1; ++k) {
    const int sk1 = inc(sk), sk2 = inc(sk1), skm = sk == 0 ? kPRing - 1 : sk - 1;   // planes k+1, k+2, k-1
    // global words this step needs, issued first: the next cell's flags and the
    // patch-row bits of this node's w rows
    const unsigned int f2 = flag_of(k + 2);
    const bool wk = do_w && k >= k0 && do_dot;
    const int ex_e = ex0 + k * exs, ey_e = ey0 + k * eys, ez_e = ez0 + k * ezs;
    const unsigned int bwx = (wk && I < nx) ? tb.pbits[ex_e >> 5] : 0u;
    const unsigned int bwy = (wk && J < ny) ? tb.pbits[ey_e >> 5] : 0u;
    const unsigned int bwz = (wk && k < nz) ? tb.pbits[ez_e >> 5] : 0u;
    // ---- vc(I, J, k+1) from the staged planes k+1, k+2 ---------------------------
    ap[0] = ap[1] = ap[2] = 0.0;
    if (cell_in(k + 1)) {
      const int c = ccol + (k + 1) * cplane;
      if (f1 & kFlagExactVc) {
        ap[0] = vcm[c]; ap[1] = vcm[nc + c]; ap[2] = vcm[2 * nc + c];
      } else {
        vc_staged(ring + sk1 * kPPlane, ring + sk2 * kPPlane, tx, ty, s_a, ap[0], ap[1], ap[2]);
      }
    }
    const int sl = (k + 1) & 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) s_vc[sl][d][ty][tx] = ap[d];
    __syncthreads();
    // plane k+4 into the ring slot of plane k-1 (last read before this barrier)
    load_p_plane(l, p, ring + skm * kPPlane, s_poff, k + 4, tid);
    cp_async_commit();
    // ---- vq(I, J, k) ---------------------------------------------------------------
    double xp[3], xm[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      xp[d] = __shfl_down_sync(0xffffffffu, a0[d], 1);
      xm[d] = __shfl_up_sync(0xffffffffu, a0[d], 1);
    }
    if (do_vq) {
      double q[3] = {0.0, 0.0, 0.0};
      if (cell_in(k)) {
        const int c = ccol + k * cplane;
        if (f0 & kFlagExactVq) {
          q[0] = vq[c];
          q[1] = vq[nc + c];
          q[2] = vq[2 * nc + c];
        } else {
          const int s0 = k & 1;
          const bool xpn = I + 1 < nx, xmn = I > 0, ypn = J + 1 < ny, ymn = J > 0, zpn = k + 1 < nz, zmn = k > 0;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double x0v = a0[d];
            double acc = 0;
            acc += xpn ? xp[d] - x0v : -2 * x0v;
            acc += xmn ? xm[d] - x0v : -2 * x0v;
            acc += ypn ? s_vc[s0][d][ty + 1][tx] - x0v : -2 * x0v;
            acc += ymn ? s_vc[s0][d][ty - 1][tx] - x0v : -2 * x0v;
            acc += zpn ? ap[d] - x0v : -2 * x0v;
            acc += zmn ? am[d] - x0v : -2 * x0v;
            q[d] = rou * x0v - kf * (acc * inv_h2);
          }
          // the exact w rows of k_patchRI read this cell's vq: the owner stores it
          if (own && k >= k0 && (f0 & kFlagStoreVq)) {
            vq[c] = q[0];
            vq[nc + c] = q[1];
            vq[2 * nc + c] = q[2];
          }
        }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) s_vq[d][ty][tx] = q[d];
    }
    cp_async_wait<1>();   // this thread's copies of plane k+3 have landed
    __syncthreads();
    // ---- w on node plane k (ri_plane with vq from shared memory) ---------------------
    if (k >= k0) {
      double dot = 0.0;
      if (do_w) {
        const int i = I, j = J;
        const bool c00 = i < nx && j < ny, cm0 = i > 0 && i <= nx && j < ny, c0m = i < nx && j > 0 && j <= ny,
                   cmm = i > 0 && j > 0 && i <= nx && j <= ny;
        const bool zin = k < nz;
        // p of the node's three edges from the staged plane k (the dot's left factor)
        const double* pk = ring + sk * kPPlane;
        const double px = (do_dot && i < nx) ? pk[ty * FX + tx] : 0.0;
        const double py = (do_dot && j < ny) ? pk[kPEx + ty * FPX + tx] : 0.0;
        const double pz = (do_dot && zin) ? pk[kPEx + kPEy + ty * FPX + tx] : 0.0;
        const double vz00 = (zin && c00) ? s_vq[2][ty][tx] : 0.0;
        const double vzm0 = (zin && cm0) ? s_vq[2][ty][tx - 1] : 0.0;
        const double vz0m = (zin && c0m) ? s_vq[2][ty - 1][tx] : 0.0;
        double fx = 0, fy = 0, fx_jm = 0, fy_im = 0;
        if (zin) {
          const double vx00 = c00 ? s_vq[0][ty][tx] : 0.0, vxm0 = cm0 ? s_vq[0][ty][tx - 1] : 0.0;
          const double vy00 = c00 ? s_vq[1][ty][tx] : 0.0, vy0m = c0m ? s_vq[1][ty - 1][tx] : 0.0;
          if (j < ny) fx = hh * (vxm0 + vx00);
          if (i < nx) fy = hh * (vy0m + vy00);
          if (j > 0) fx_jm = hh * ((cmm ? s_vq[0][ty - 1][tx - 1] : 0.0) + (c0m ? s_vq[0][ty - 1][tx] : 0.0));
          if (i > 0) fy_im = hh * ((cmm ? s_vq[1][ty - 1][tx - 1] : 0.0) + (cm0 ? s_vq[1][ty][tx - 1] : 0.0));
        }
        const double fz = (i < nx && j < ny) ? hh * (c_vz00 + vz00) : 0.0;
        const double fz_im = (i > 0 && j < ny) ? hh * (c_vzm0 + vzm0) : 0.0;
        const double fz_jm = (i < nx && j > 0) ? hh * (c_vz0m + vz0m) : 0.0;
        if (i < nx) {
          const double val = fz - fz_jm + c_fy - fy;
          w[ex_e] = val;
          if (!((bwx >> (ex_e & 31)) & 1u)) dot += px * val;
        }
        if (j < ny) {
          const double val = fx - c_fx + fz_im - fz;
          w[ey_e] = val;
          if (!((bwy >> (ey_e & 31)) & 1u)) dot += py * val;
        }
        if (zin) {
          const double val = fy - fy_im + fx_jm - fx;
          w[ez_e] = val;
          if (!((bwz >> (ez_e & 31)) & 1u)) dot += pz * val;
        }
        c_vz00 = vz00; c_vzm0 = vzm0; c_vz0m = vz0m;
        c_fx = fx; c_fy = fy;
      }
      if (do_dot) {
        for (int o = 16; o > 0; o >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, o);
        if (tx == 0) s_dot[k - k0][ty] = dot;
      }
    } else if (do_w) {
      // plane k0 - 1: only the carried values of node (I, J)
      const int i = I, j = J;
      const bool c00 = i < nx && j < ny, cm0 = i > 0 && i <= nx && j < ny, c0m = i < nx && j > 0 && j <= ny;
      const bool zin = k >= 0 && k < nz;
      c_vz00 = (zin && c00) ? s_vq[2][ty][tx] : 0.0;
      c_vzm0 = (zin && cm0) ? s_vq[2][ty][tx - 1] : 0.0;
      c_vz0m = (zin && c0m) ? s_vq[2][ty - 1][tx] : 0.0;
      c_fx = c_fy = 0.0;
      if (zin) {
        if (i < nx) c_fy = hh * ((c0m ? s_vq[1][ty - 1][tx] : 0.0) + (c00 ? s_vq[1][ty][tx] : 0.0));
        if (j < ny) c_fx = hh * ((cm0 ? s_vq[0][ty][tx - 1] : 0.0) + (c00 ? s_vq[0][ty][tx] : 0.0));
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      am[d] = a0[d];
      a0[d] = ap[d];
    }
    f0 = f1;
    f1 = f2;
    sk = sk1;
  }
  cp_async_wait<0>();   // no copy may still target this block's shared memory at exit
  if (!do_dot) return;
  __syncthreads();
  // one partial per (level, tile, node plane), its 16 warp sums combined in a fixed
  // order: the dot does not depend on the z-chunk depth the autotuner picked
  if (tid < k1 - k0) {
    const double* q = s_dot[tid];
    const double v = (((q[0] + q[8]) + (q[4] + q[12])) + ((q[2] + q[10]) + (q[6] + q[14]))) +
                     (((q[1] + q[9]) + (q[5] + q[13])) + ((q[3] + q[11]) + (q[7] + q[15])));
    partials[l.fplane_base + ((long long)(k0 + tid) * m.gyF + blockIdx.y) * m.gxF + blockIdx.x] = v;
  }
}

// flag byte per cell from the three bit arrays (kFlagExactVc | kFlagExactVq | kFlagStoreVq)
__global__ void k_cell_flags(long long nc, const unsigned int* __restrict__ a, const unsigned int* __restrict__ v,
                             const unsigned int* __restrict__ r, unsigned char* flags) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc;
       c += (long long)gridDim.x * blockDim.x) {
    unsigned int f = 0;
    if (bit_set(a, c)) f |= kFlagExactVc;
    if (bit_set(v, c)) f |= kFlagExactVq;
    if (bit_set(r, c)) f |= kFlagStoreVq;
    flags[c] = (unsigned char)f;
  }
}

// template vc of listed regular cells whose vc an exact V row reads (k_patchV)
__global__ void __launch_bounds__(kThreads) k_vc_list(Meta m, long long n, const int* __restrict__ cells,
                                                      const double* __restrict__ p, double* vcm,
                                                      const CGState* __restrict__ st) {
  if (st->done) return;
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int c = cells[q];
  int L = 0;
  while (L + 1 < m.nl && c >= m.lv[L + 1].cbase) ++L;
  const LevelMeta& l = m.lv[L];
  const int loc = c - (int)l.cbase;
  const int i = loc % l.n[0], j = (loc / l.n[0]) % l.n[1], k = loc / (l.n[0] * l.n[1]);
  double vx, vy, vz;
  vc_template(l, p, i, j, k, vx, vy, vz);
  vcm[c] = vx;
  vcm[m.nc + c] = vy;
  vcm[2 * m.nc + c] = vz;
}

// setup: flags[c] |= bit for the listed cells
__global__ void k_flag_list(long long n, const int* __restrict__ ids, long long nc, unsigned char bit,
                            unsigned char* flags) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int c = ids[q];
    if (c >= 0 && c < nc) flags[c] |= bit;
  }
}

// setup: cell bits from a list of cell ids (or of component-major vq columns)
__global__ void k_mark_cells(long long n, const int* __restrict__ ids, long long nc, unsigned int* bits) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    long long c = ids[q];
    c %= nc;
    atomicOr(&bits[c >> 5], 1u << (c & 31));
  }
}

// ---------------------------------------------------------------------------
// CG vector kernels (float64 state, T = working type of p/w)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_cg_init(long long ne, const double* __restrict__ res_e,
                                                      const double* __restrict__ s,
                                                      const double* __restrict__ prec, double* x,
                                                      double* r, double* p, double* partials,
                                                      CGState* st) {
  double v[3] = {0.0, 0.0, 0.0};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const double pr = prec[e];
    const double re = pr != 0.0 ? res_e[e] : 0.0;
    const double xe = s[e];
    r[e] = re;
    x[e] = xe;
    const double pe = re * pr;
    p[e] = pe;
    v[0] += re * re;
    v[1] += pe * re;
    v[2] += xe * xe;
  }
  if (grid_sum<3>(v, partials, &st->counter) && threadIdx.x == 0) {
    st->l2_0 = v[0];
    st->eta = v[1];
    st->xnorm = v[2] + 1e-16;
    st->thresh = st->xnorm * (st->tol1 * st->tol1) + (st->tol2 * st->tol2) * v[1];
    st->m = 0;
    st->done = 0;
    st->iters = 0;
    st->stop = 0;
  }
}

// Preconditioner value of edge e: the level's regular value unless the edge is flagged.
__device__ __forceinline__ double prec_of(const Meta& m, const unsigned int* __restrict__ bits,
                                          const double* __restrict__ prec, long long e) {
  if (bit_set(bits, e)) return prec[e];
  int L = 0;
  while (L + 1 < m.nl && e >= m.lv[L + 1].ebase[0]) ++L;
  return m.lv[L].prec_reg;
}

// r -= alpha w on unmasked edges; eta' = sum (r*prec)*r; the last block applies the
// stopping test (every `check` iterations, or at cg_max) and sets `stop`.
__device__ __forceinline__ void cg_update_blocks(Grid1 g, const Meta& m, long long ne, double* r,
                                                 const double* __restrict__ w,
                                                 const unsigned int* __restrict__ pbits,
                                                 const double* __restrict__ prec, double* partials, CGState* st) {
  const double alpha = st->alpha;
  double v[1] = {0.0};
  // two elements of the thread's grid-stride sequence per pass, loads first (more
  // bytes in flight); each element is computed and summed in the original order
  const long long S = (long long)g.nb * blockDim.x;
  long long e = g.b * (long long)blockDim.x + threadIdx.x;
  for (; e + S < ne; e += 2 * S) {
    double pr[2], rv[2], wv[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      pr[u] = prec_of(m, pbits, prec, e + u * S);
      rv[u] = r[e + u * S];
      wv[u] = w[e + u * S];
    }
#pragma unroll
    for (int u = 0; u < 2; ++u)
      if (pr[u] != 0.0) {
        const double re = rv[u] - alpha * wv[u];
        r[e + u * S] = re;
        v[0] += (re * pr[u]) * re;
      }
  }
  for (; e < ne; e += S) {
    const double pr = prec_of(m, pbits, prec, e);
    if (pr != 0.0) {
      const double re = r[e] - alpha * w[e];
      r[e] = re;
      v[0] += (re * pr) * re;
    }
  }
  if (grid_sum_at<1>(v, partials, &st->counter, g.b, g.nb)) {
    const double en = v[0];
    st->eta_new = en;
    const int mm = st->m + 1;
    st->m = mm;
    bool stop = false;
    if (mm % st->check == 0) {
      if (!isfinite(en) || en < st->thresh) stop = true;
    }
    if (mm >= st->cg_max) stop = true;
    if (stop) {
      st->stop = 1;
      st->iters = mm;
    } else {
      st->beta = en / (st->eta != 0.0 ? st->eta : INFINITY);
      st->eta = en;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 8) k_cg_update(Meta m, long long ne, double* r,
                                                        const double* __restrict__ w,
                                                        const unsigned int* __restrict__ pbits,
                                                        const double* __restrict__ prec,
                                                        double* partials, CGState* st) {
  if (st->done) return;
  cg_update_blocks(own_grid1(), m, ne, r, w, pbits, prec, partials, st);
}

// x += alpha p (the iterate of this iteration), then p = r*prec + beta p unless the
// stopping test fired; the last block turns `stop` into `done`.
__device__ __forceinline__ void cg_p_blocks(Grid1 g, const Meta& m, long long ne, const double* __restrict__ r,
                                            const unsigned int* __restrict__ pbits,
                                            const double* __restrict__ prec, double* p, double* x, CGState* st) {
  const double alpha = st->alpha, beta = st->beta;
  const bool stop = st->stop != 0;
  for (long long e = g.b * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)g.nb * blockDim.x) {
    const double pe = p[e];
    x[e] += alpha * pe;
    if (!stop) p[e] = r[e] * prec_of(m, pbits, prec, e) + beta * pe;
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int t = atomicAdd(&st->counter2, 1u);
    last = (t == (unsigned int)g.nb - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    st->counter2 = 0u;
    if (stop) st->done = 1;
  }
}

__global__ void __launch_bounds__(kThreads) k_cg_p(Meta m, long long ne, const double* __restrict__ r,
                                                   const unsigned int* __restrict__ pbits,
                                                   const double* __restrict__ prec, double* p, double* x,
                                                   CGState* st) {
  if (st->done) return;
  cg_p_blocks(own_grid1(), m, ne, r, pbits, prec, p, x, st);
}

__global__ void k_mask(long long n, const double* __restrict__ prec, double* w) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    if (prec[e] == 0.0) w[e] = 0.0;
}

__global__ void k_sub(long long n, const double* a, const double* b, double* out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    out[e] = a[e] - b[e];
}

// true residual: tr = (res_e - A d) masked; eta = sum tr*prec*tr, l2 = sum tr^2
__global__ void __launch_bounds__(kThreads) k_cg_true(long long ne, const double* __restrict__ res_e,
                                                      const double* __restrict__ Ad,
                                                      const double* __restrict__ prec,
                                                      int use_Ad, double* partials, CGState* st) {
  double v[2] = {0.0, 0.0};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const double pr = prec[e];
    if (pr == 0.0) continue;
    const double tr = use_Ad ? res_e[e] - Ad[e] : res_e[e];
    v[0] += (tr * pr) * tr;
    v[1] += tr * tr;
  }
  if (grid_sum<2>(v, partials, &st->counter) && threadIdx.x == 0) {
    st->true_eta = v[0];
    st->true_l2 = v[1];
  }
}

// ---------------------------------------------------------------------------
// mixed precision: float32 PCG inside float64 iterative refinement
// ---------------------------------------------------------------------------
__global__ void k_d2f(long long n, const double* __restrict__ a, float* b) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    b[e] = (float)a[e];
}

// inner start: r32 = r64 (masked), d32 = 0, p32 = r32*dinv, eta = sum (r32*dinv)*r32
__global__ void __launch_bounds__(kThreads) k_mix_start(long long ne, const double* __restrict__ r64,
                                                        const float* __restrict__ dinv, float* r32,
                                                        float* d32, float* p32, double eps_in2,
                                                        double* partials, CGState* st) {
  double v[1] = {0.0};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const float di = dinv[e];
    const float re = di != 0.f ? (float)r64[e] : 0.f;
    r32[e] = re;
    d32[e] = 0.f;
    const float pe = re * di;
    p32[e] = pe;
    v[0] += (double)pe * (double)re;
  }
  if (grid_sum<1>(v, partials, &st->counter)) {
    st->eta = v[0];
    st->thresh_in = eps_in2 * v[0];
    st->m = 0;
    st->done = v[0] > 0.0 ? 0 : 1;
    st->iters = 0;
  }
}

__device__ __forceinline__ void cg_update32_blocks(Grid1 g, long long ne, float* d32, float* r32,
                                                   const float* __restrict__ p32, const float* __restrict__ w32,
                                                   const float* __restrict__ dinv, double* partials, CGState* st) {
  const float alpha = (float)st->alpha;
  double v[1] = {0.0};
  for (long long e = g.b * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)g.nb * blockDim.x) {
    const float di = dinv[e];
    if (di != 0.f) {
      d32[e] += alpha * p32[e];
      const float re = r32[e] - alpha * w32[e];
      r32[e] = re;
      v[0] += (double)(re * di) * (double)re;
    }
  }
  if (grid_sum_at<1>(v, partials, &st->counter, g.b, g.nb)) {
    const double en = v[0];
    const int m = st->m + 1;
    st->m = m;
    bool stop = false;
    if (m % st->check == 0 && (!isfinite(en) || en < st->thresh_in)) stop = true;
    if (m >= st->cg_max) stop = true;
    if (stop) {
      st->done = 1;
      st->iters = m;
    } else {
      st->beta = en / (st->eta != 0.0 ? st->eta : INFINITY);
      st->eta = en;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_cg_update32(long long ne, float* d32, float* r32,
                                                          const float* __restrict__ p32,
                                                          const float* __restrict__ w32,
                                                          const float* __restrict__ dinv,
                                                          double* partials, CGState* st) {
  if (st->done) return;
  cg_update32_blocks(own_grid1(), ne, d32, r32, p32, w32, dinv, partials, st);
}

__device__ __forceinline__ void cg_p32_blocks(Grid1 g, long long ne, const float* __restrict__ r32,
                                              const float* __restrict__ dinv, float* p32, const CGState* st) {
  const float beta = (float)st->beta;
  const long long S = (long long)g.nb * blockDim.x;
  long long e = g.b * (long long)blockDim.x + threadIdx.x;
  for (; e + 3 * S < ne; e += 4 * S) {
    float rv[4], dv[4], pv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      rv[u] = r32[e + u * S];
      dv[u] = dinv[e + u * S];
      pv[u] = p32[e + u * S];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) p32[e + u * S] = rv[u] * dv[u] + beta * pv[u];
  }
  for (; e < ne; e += S) p32[e] = r32[e] * dinv[e] + beta * p32[e];
}

__global__ void __launch_bounds__(kThreads, 8) k_cg_p32(long long ne, const float* __restrict__ r32,
                                                     const float* __restrict__ dinv, float* p32,
                                                     const CGState* st) {
  if (st->done) return;
  cg_p32_blocks(own_grid1(), ne, r32, dinv, p32, st);
}

// Reliable update of the float32 CG: r32 = float(r64) (the float64 residual after
// folding the float32 correction into x), correction reset, eta from the new residual,
// beta = eta_new / eta_old so that k_cg_p32 continues the same search direction.
__global__ void __launch_bounds__(kThreads) k_mix_reliable(long long ne, const double* __restrict__ r64,
                                                           const float* __restrict__ dinv, float* r32,
                                                           float* d32, double eps_in2, double* partials,
                                                           CGState* st) {
  double v[1] = {0.0};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const float di = dinv[e];
    const float re = di != 0.f ? (float)r64[e] : 0.f;
    r32[e] = re;
    d32[e] = 0.f;
    v[0] += (double)(re * di) * (double)re;
  }
  if (grid_sum<1>(v, partials, &st->counter)) {
    const double en = v[0];
    st->beta = en / (st->eta != 0.0 ? st->eta : INFINITY);
    st->eta = en;
    st->thresh_in = eps_in2 * en;
    st->m = 0;
    st->iters = 0;
    st->done = en > 0.0 && isfinite(en) ? 0 : 1;
  }
}

// d = double(x32) on unmasked edges (0 elsewhere): the float32 correction in float64
__global__ void k_mix_widen(long long ne, const float* __restrict__ x32, double* d,
                            const double* __restrict__ prec) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x)
    d[e] = prec[e] != 0.0 ? (double)x32[e] : 0.0;
}

// x += d; r -= q on unmasked edges; true_eta = sum (r*prec)*r, true_l2 = sum r^2
__global__ void __launch_bounds__(kThreads) k_mix_fold(long long ne, const double* __restrict__ d,
                                                       const double* __restrict__ q, double* x, double* r,
                                                       const double* __restrict__ prec, double* partials,
                                                       CGState* st) {
  double v[2] = {0.0, 0.0};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const double pr = prec[e];
    x[e] += d[e];
    if (pr != 0.0) {
      const double re = r[e] - q[e];
      r[e] = re;
      v[0] += (re * pr) * re;
      v[1] += re * re;
    }
  }
  if (grid_sum<2>(v, partials, &st->counter)) {
    st->true_eta = v[0];
    st->true_l2 = v[1];
  }
}

// diagonal probing: p = 1 on the edges of one colour (level L, axis a, index residues mod q)
__global__ void k_probe_set(long long ne, long long base, int dx, int dy, int cnt, int q, int ci, int cj,
                            int ck, double* p, int clear) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    double v = 0.0;
    const long long loc = e - base;
    if (loc >= 0 && loc < cnt && !clear) {
      const int l = (int)loc;
      const int i = l % dx, j = (l / dx) % dy, k = l / (dx * dy);
      if (i % q == ci && j % q == cj && k % q == ck) v = 1.0;
    }
    p[e] = v;
  }
}

__global__ void k_probe_get(long long base, int dx, int dy, int cnt, int q, int ci, int cj, int ck,
                            const double* __restrict__ w, double* diag) {
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < cnt; l += gridDim.x * blockDim.x) {
    const int i = l % dx, j = (l / dx) % dy, k = l / (dx * dy);
    if (i % q == ci && j % q == cj && k % q == ck) diag[base + l] = w[base + l];
  }
}

// dinv = 1/(rou*diag1 + kfac*diag2) on unmasked edges, 0 elsewhere
__global__ void k_dinv(long long ne, const double* __restrict__ d1, const double* __restrict__ d2,
                       const double* __restrict__ prec, double rou, double kfac, float* dinv) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const double d = rou * d1[e] + kfac * d2[e];
    dinv[e] = (prec[e] != 0.0 && d > 0.0) ? (float)(1.0 / d) : 0.f;
  }
}

// ---------------------------------------------------------------------------
// Batched CG iterations: every stage of one iteration (matvec kernels A, V, RI with
// their exact rows, the residual update and the direction update) is one launch over
// the tiles of all cases of a batch.  Block b of a stage reads blk[b] = (case, block
// within that case's grid) and runs the single-case body with those coordinates, so
// every case computes exactly what its own kernels compute.  A case whose solve has
// stopped (st->done) leaves its blocks idle; the host drops it from the tables.
// ---------------------------------------------------------------------------
constexpr int kBStages = 8;
constexpr int kBatchCellDepth = 16, kBatchNodeDepth = 16;   // z planes of a batched cell / node tile
constexpr int kBatchGroups = 16;  // cost-balanced groups of cases, parallel branches of the chunk graph

struct BCase {
  Meta m;                          // the case's layout decoding and tiles, of the batch's precision
  CGState* st;
  double* partials;
  void *p, *w, *vcm, *vq, *r, *x;  // the CG vectors in the batch's precision (x: the float32 correction)
  const void *pa_val, *pv_val, *pr_val;
  const int *pa_ids, *pa_col, *pv_ids, *pv_col, *pr_ids, *pr_col;
  const long long *pa_ptr, *pv_ptr, *pr_ptr;
  const unsigned int *prec_bits, *pr_bits;
  const double* prec;              // float64 preconditioner exceptions
  const float* dinv;               // float32 Jacobi (mixed solver)
  long long nA, nV, nR, ne, nc;
  int nblk[kBStages];              // the case's blocks in each stage (its single-case grids)
};

__device__ __forceinline__ Grid3 batch_grid3(int lb, int gx, int gy, int gz) {
  return Grid3{lb % gx, (lb / gx) % gy, lb / (gx * gy), gx, gy, gz};
}

template <typename T>
__global__ void __launch_bounds__(TX * TY) k_bA(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  const Meta& m = q.m;
  mvA_tile<T>(m, batch_grid3(cb.y, m.gxA, m.gyA, m.gzA), (const T*)q.p, (T*)q.vcm);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_bpatchA(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  patchA_rows<T>(Grid1{cb.y, q.nblk[1]}, q.nA, q.pa_ids, q.pa_ptr, q.pa_col, (const T*)q.pa_val, (const T*)q.p,
                 (T*)q.vcm, q.nc);
}

template <typename T>
__global__ void __launch_bounds__(TX * TY, 4) k_bV(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  const Meta& m = q.m;
  mvV_tile<T>(m, batch_grid3(cb.y, m.gxV, m.gyA, m.gzA), (const T*)q.vcm, (T*)q.vq, q.st);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_bpatchV(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  patchV_rows<T>(Grid1{cb.y, q.nblk[3]}, q.nV, q.pv_ids, q.pv_ptr, q.pv_col, (const T*)q.pv_val,
                 (const T*)q.vcm, (T*)q.vq, q.nc, q.st);
}

template <typename T>
__global__ void __launch_bounds__(TX * TY) k_bRI(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  const Meta& m = q.m;
  mvRI_tile<T>(m, batch_grid3(cb.y, m.gxR, m.gyR, m.gzR), (const T*)q.vq, (T*)q.w, (const T*)q.p, q.pr_bits,
               q.partials, 1);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_bpatchRI(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  patchRI_rows<T>(Grid1{cb.y, q.nblk[5]}, q.nR, q.pr_ids, q.pr_ptr, q.pr_col, (const T*)q.pr_val,
                  (const T*)q.vq, (T*)q.w, (const T*)q.p, q.partials, q.m.nplanes, q.st, 1);
}

// float64 residual update and direction (k_cg_update, k_cg_p)
__global__ void __launch_bounds__(kThreads, 8) k_bupdate(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  cg_update_blocks(Grid1{cb.y, q.nblk[6]}, q.m, q.ne, (double*)q.r, (const double*)q.w, q.prec_bits, q.prec,
                   q.partials, q.st);
}

__global__ void __launch_bounds__(kThreads, 8) k_bdir(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  cg_p_blocks(Grid1{cb.y, q.nblk[7]}, q.m, q.ne, (const double*)q.r, q.prec_bits, q.prec, (double*)q.p,
              (double*)q.x, q.st);
}

// float32 residual update and direction of the mixed solver (k_cg_update32, k_cg_p32)
__global__ void __launch_bounds__(kThreads, 8) k_bupdate32(const BCase* __restrict__ cs,
                                                           const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  cg_update32_blocks(Grid1{cb.y, q.nblk[6]}, q.ne, (float*)q.x, (float*)q.r, (const float*)q.p,
                     (const float*)q.w, q.dinv, q.partials, q.st);
}

__global__ void __launch_bounds__(kThreads, 8) k_bdir32(const BCase* __restrict__ cs, const int2* __restrict__ blk) {
  const int2 cb = blk[blockIdx.x];
  const BCase& q = cs[cb.x];
  if (q.st->done) return;
  cg_p32_blocks(Grid1{cb.y, q.nblk[7]}, q.ne, (const float*)q.r, q.dinv, (float*)q.p, q.st);
}

struct GState {
  double rz, rr, bb, atol, alpha, beta;
  unsigned int counter;
  int done, iters;
};

// The stop test of scipy.sparse.linalg.cg (atol = 0): |r| < rtol |b|, checked
// before every iteration; once it holds every kernel below returns at once, so
// chunks of launches may run past convergence without changing x.
__global__ void __launch_bounds__(kThreads) k_g_init(long long n, double rtol, const double* __restrict__ b,
                                                     const double* __restrict__ dinv, double* x, double* r,
                                                     double* z, double* p, double* partials, GState* g) {
  double v[2] = {0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double bi = b[i], zi = dinv[i] * bi;
    x[i] = 0.0; r[i] = bi; z[i] = zi; p[i] = zi;
    v[0] += bi * zi;
    v[1] += bi * bi;
  }
  if (grid_sum<2>(v, partials, &g->counter)) {
    g->rz = v[0]; g->bb = v[1]; g->rr = v[1];
    g->atol = rtol * sqrt(v[1]);
    g->iters = 0;
    g->done = v[1] == 0.0 || sqrt(v[1]) < g->atol;
  }
}

// q = A p and the p.q sum for alpha in one pass (one row per thread); the
// thread-to-row map and the order of the sums are those of a separate p.q kernel
// on the same grid.
__global__ void __launch_bounds__(kThreads) k_g_mvpq(long long n, const long long* __restrict__ ptr,
                                                     const int* __restrict__ col, const double* __restrict__ val,
                                                     const double* __restrict__ p, double* __restrict__ q,
                                                     double* partials, GState* g) {
  if (g->done) return;
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double acc = csr_row<double>(ptr, col, val, p, i);
    q[i] = acc;
    v[0] += p[i] * acc;
  }
  if (grid_sum<1>(v, partials, &g->counter)) g->alpha = v[0] != 0.0 ? g->rz / v[0] : 0.0;
}

__global__ void __launch_bounds__(kThreads) k_g_update(long long n, const double* __restrict__ p,
                                                       const double* __restrict__ q, const double* __restrict__ dinv,
                                                       double* x, double* r, double* z, double* partials, GState* g) {
  if (g->done) return;
  const double a = g->alpha;
  double v[2] = {0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += a * p[i];
    const double ri = r[i] - a * q[i];
    r[i] = ri;
    const double zi = dinv[i] * ri;
    z[i] = zi;
    v[0] += ri * zi;
    v[1] += ri * ri;
  }
  if (grid_sum<2>(v, partials, &g->counter)) {
    g->beta = g->rz != 0.0 ? v[0] / g->rz : 0.0;
    g->rz = v[0];
    g->rr = v[1];
    g->iters += 1;
    if (sqrt(v[1]) < g->atol) g->done = 1;
  }
}

__global__ void k_g_p(long long n, const double* __restrict__ z, double* p, const GState* g) {
  if (g->done) return;
  const double b = g->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = z[i] + b * p[i];
}


// ---------------------------------------------------------------------------
// Offline pressure recovery on the device (ib_postprocess.py:49-107): input
// checks, the face weights and jumps, the Laplacian in CSR (cell 0 pinned: its
// row is empty and rhs[0] = dinv[0] = 0, so p[0] stays 0 and its column adds
// exact zeros), a reachability sweep for the connectivity check, the gauge and
// the projection residual.  Sums are in fixed orders: per-row sums follow the
// sorted (neighbour, face) keys, grid sums follow the block order.
// ---------------------------------------------------------------------------
enum : unsigned { kPrPos = 1u, kPrGrad = 2u, kPrIds = 4u, kPrAreaNf = 8u, kPrAreaNeg = 16u, kPrDist = 32u };

struct PrState {
  unsigned int err;
  unsigned int counter;
  unsigned long long reached;
};

__global__ void k_pr_cells(long long n3, const double* __restrict__ pos, const double* __restrict__ grad,
                           PrState* st) {
  unsigned int e = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x) {
    if (!isfinite(pos[i])) e |= kPrPos;
    if (!isfinite(grad[i])) e |= kPrGrad;
  }
  if (e) atomicOr(&st->err, e);
}

// per face: ids checked before any use; internal faces get w = A/|d| and the jump
// 0.5 (g1 + g2).d, summed in the reference's component order
__global__ void k_pr_faces(long long nf, long long n, const long long* __restrict__ pairs,
                           const double* __restrict__ area, const double* __restrict__ pos,
                           const double* __restrict__ grad, unsigned int* deg, double* w_f, double* jump_f,
                           unsigned char* bflag, PrState* st) {
  unsigned int e = 0;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
    const long long a = pairs[2 * f], b = pairs[2 * f + 1];
    w_f[f] = 0.0;
    jump_f[f] = 0.0;
    if (a < 0 || a >= n || b < -1 || b >= n) { e |= kPrIds; continue; }
    const double ar = area[f];
    if (!isfinite(ar)) e |= kPrAreaNf;
    else if (!(ar > 0.0)) e |= kPrAreaNeg;
    if (b < 0) { bflag[a] = 1; continue; }
    const double dx = pos[3 * b] - pos[3 * a], dy = pos[3 * b + 1] - pos[3 * a + 1], dz = pos[3 * b + 2] - pos[3 * a + 2];
    const double dist = sqrt((dx * dx + dy * dy) + dz * dz);
    if (!(dist > 0.0)) { e |= kPrDist; continue; }
    const double s0 = (grad[3 * a] + grad[3 * b]) * dx, s1 = (grad[3 * a + 1] + grad[3 * b + 1]) * dy,
                 s2 = (grad[3 * a + 2] + grad[3 * b + 2]) * dz;
    const double w = ar / dist;
    w_f[f] = w;
    jump_f[f] = 0.5 * ((s0 + s1) + s2);
    if (w > 0.0) {                 // the same test as k_pr_fill: one key per count
      atomicAdd(&deg[a], 1u);
      atomicAdd(&deg[b], 1u);
    }
  }
  if (e) atomicOr(&st->err, e);
}

// key lengths per row (row 0 pinned: none); klen has n + 1 entries, the last 0
__global__ void k_pr_klen(long long n, const unsigned int* __restrict__ deg, int* klen) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c <= n; c += (long long)gridDim.x * blockDim.x)
    klen[c] = (c == 0 || c == n) ? 0 : (int)deg[c];
}

// key = (neighbour << 32) | (face << 1) | side, side 1 when the row's cell is the face's second cell
__global__ void k_pr_fill(long long nf, const long long* __restrict__ pairs, const double* __restrict__ w_f,
                          int* kcur, unsigned long long* keys) {
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
    const long long a = pairs[2 * f], b = pairs[2 * f + 1];
    if (b < 0 || !(w_f[f] > 0.0)) continue;
    const unsigned long long lo = (unsigned long long)f << 1;
    if (a != 0) keys[atomicAdd(&kcur[a], 1)] = ((unsigned long long)b << 32) | lo;
    if (b != 0) keys[atomicAdd(&kcur[b], 1)] = ((unsigned long long)a << 32) | lo | 1ull;
  }
}

// one row per thread: diagonal first, then the neighbours in key order
__global__ void k_pr_rows(long long n, const int* __restrict__ kptr, const unsigned long long* __restrict__ keys,
                          const double* __restrict__ w_f, const double* __restrict__ jump_f, long long* ptr, int* col,
                          double* val, double* rhs, double* dinv) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (c == n - 1) ptr[n] = (long long)kptr[n] + (n - 1);
    if (c == 0) {
      ptr[0] = 0;
      rhs[0] = 0.0;
      dinv[0] = 0.0;
      continue;
    }
    const long long base = (long long)kptr[c] + (c - 1);
    ptr[c] = base;
    double diag = 0.0, sum = 0.0;
    long long o = base + 1;
    for (int k = kptr[c]; k < kptr[c + 1]; ++k, ++o) {
      const unsigned long long key = keys[k];
      const long long f = (long long)((key & 0xffffffffull) >> 1);
      const double w = w_f[f], wj = w * jump_f[f];
      diag += w;
      sum += (key & 1ull) ? wj : -wj;
      col[o] = (int)(key >> 32);
      val[o] = -w;
    }
    col[base] = (int)c;
    val[base] = diag;
    rhs[c] = sum;
    dinv[c] = diag > 0.0 ? 1.0 / diag : 0.0;
  }
}

// cells reachable from cell 0: a cell joins when a neighbour in its row has
// joined (monotone, so concurrent sweeps only speed it up)
__global__ void __launch_bounds__(kThreads) k_pr_reach(long long n, const long long* __restrict__ ptr,
                                                       const int* __restrict__ col, volatile unsigned char* vis,
                                                       PrState* st) {
  __shared__ unsigned int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  unsigned int mine = 0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (vis[c]) continue;
    for (long long k = ptr[c] + 1; k < ptr[c + 1]; ++k)
      if (vis[col[k]]) {
        vis[c] = 1;
        ++mine;
        break;
      }
  }
  if (mine) atomicAdd(&cnt, mine);
  __syncthreads();
  if (threadIdx.x == 0 && cnt) atomicAdd(&st->reached, (unsigned long long)cnt);
}

__global__ void __launch_bounds__(kThreads) k_pr_gauge(long long n, const double* __restrict__ x,
                                                       const unsigned char* __restrict__ bflag, double* partials,
                                                       unsigned int* counter, double* out) {
  double v[3] = {0.0, 0.0, 0.0};
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const double xc = x[c];
    if (bflag[c]) { v[0] += xc; v[1] += 1.0; }
    v[2] += xc;
  }
  if (grid_sum<3>(v, partials, counter)) { out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; }
}

__global__ void k_pr_shift(long long n, double* x, double mean) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    x[c] -= mean;
}

__global__ void __launch_bounds__(kThreads) k_pr_mismatch(long long nf, const long long* __restrict__ pairs,
                                                          const double* __restrict__ x, const double* __restrict__ w_f,
                                                          const double* __restrict__ jump_f, double* partials,
                                                          unsigned int* counter, double* out) {
  double v[2] = {0.0, 0.0};
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
    const long long b = pairs[2 * f + 1];
    if (b < 0) continue;
    const double w = w_f[f], m = (x[b] - x[pairs[2 * f]]) - jump_f[f];
    v[0] += w * (m * m);
    v[1] += w;
  }
  if (grid_sum<2>(v, partials, counter)) { out[0] = v[0]; out[1] = v[1]; }
}

// ---------------------------------------------------------------------------
// generic CSR gathers (step operators)
// ---------------------------------------------------------------------------
__global__ void k_csr(long long nrows, const long long* __restrict__ ptr, const int* __restrict__ col,
                      const double* __restrict__ val, const double* __restrict__ x, double* y) {
  for (long long rI = blockIdx.x * (long long)blockDim.x + threadIdx.x; rI < nrows;
       rI += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (long long q = ptr[rI]; q < ptr[rI + 1]; ++q) acc += val[q] * x[col[q]];
    y[rI] = acc;
  }
}

// y_d[row] = sum val3[q][d] * x[col]  (interp_f2c: rows cells, cols faces)
__global__ void k_csr_to3(long long nrows, long long ystride, const long long* __restrict__ ptr,
                          const int* __restrict__ col, const double* __restrict__ val3,
                          const double* __restrict__ x, double* y) {
  for (long long rI = blockIdx.x * (long long)blockDim.x + threadIdx.x; rI < nrows;
       rI += (long long)gridDim.x * blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (long long q = ptr[rI]; q < ptr[rI + 1]; ++q) {
      const double xv = x[col[q]];
      a0 += val3[3 * q] * xv;
      a1 += val3[3 * q + 1] * xv;
      a2 += val3[3 * q + 2] * xv;
    }
    y[rI] = a0;
    y[ystride + rI] = a1;
    y[2 * ystride + rI] = a2;
  }
}

// y[row] = sum_q sum_d val3[q][d] * x_d[col]  (integr_c2f: rows faces, cols cells)
__global__ void k_csr_from3(long long nrows, long long xstride, const long long* __restrict__ ptr,
                            const int* __restrict__ col, const double* __restrict__ val3,
                            const double* __restrict__ x, double* y) {
  for (long long rI = blockIdx.x * (long long)blockDim.x + threadIdx.x; rI < nrows;
       rI += (long long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (long long q = ptr[rI]; q < ptr[rI + 1]; ++q) {
      const long long c = col[q];
      const double t = (x[c] * val3[3 * q] + x[xstride + c] * val3[3 * q + 1]) +
                       x[2 * xstride + c] * val3[3 * q + 2];
      acc += t;
    }
    y[rI] = acc;
  }
}

__global__ void k_set_idx(long long n, const int* __restrict__ idx, const double* __restrict__ val,
                          double* y) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    y[idx[q]] = val[q];
}

// ghost cells on boundary faces (Driver.calc_vel, ib_driver_np.py:275-291)
// info: bits 0-1 axis, bit 2 inlet family, bit 3 cavity
__global__ void k_ghost(long long nbf, long long ncx, long long nc, const int* __restrict__ bf_face,
                        const int* __restrict__ bf_cell, const int* __restrict__ bf_info,
                        const double* __restrict__ bf_af, const double* __restrict__ U, double* vc) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nbf;
       b += (long long)gridDim.x * blockDim.x) {
    const int c = bf_cell[b], info = bf_info[b], a = info & 3;
    const long long g = nc + b;
    double v1[3] = {vc[c], vc[ncx + c], vc[2 * ncx + c]};
    double gv[3];
    if (info & 8) {
      gv[0] = -v1[0]; gv[1] = -v1[1]; gv[2] = -v1[2];
    } else {
      const double Af = bf_af[b], Uf = U[bf_face[b]];
      const double a2 = Af * Af;
      if (info & 4) {
        gv[0] = gv[1] = gv[2] = 0.0;
        gv[a] = (Uf * Af) / a2;
      } else {
        const double dotv = v1[a] * Af;
        gv[0] = v1[0]; gv[1] = v1[1]; gv[2] = v1[2];
        gv[a] = v1[a] + ((Uf - dotv) * Af) / a2;
      }
    }
    vc[g] = gv[0];
    vc[ncx + g] = gv[1];
    vc[2 * ncx + g] = gv[2];
  }
}

// convection + diffusion, optionally assembled into the momentum residual.
// mode 0: conv -> out0, diff -> out1 (test)
// mode 1: res0 = rou vc - c1 conv + c2 diff  (ib_driver_np.py:458)
// mode 2: res = res0 - rou vc - c1 conv + c2 diff + dt fE  (ib_driver_np.py:466-470)
__global__ void k_convdiff(long long nc, long long ncx, const long long* __restrict__ cf_ptr,
                           const int* __restrict__ cf_face, const int* __restrict__ f_lo,
                           const int* __restrict__ f_hi, const double* __restrict__ aol,
                           const double* __restrict__ volci, const double* __restrict__ U,
                           const double* __restrict__ vc, double visc, int mode, double rou,
                           double c1, double c2, double dt, const double* __restrict__ res0,
                           const double* __restrict__ fE, double* out0, double* out1) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc;
       c += (long long)gridDim.x * blockDim.x) {
    double cv[3] = {0.0, 0.0, 0.0}, df[3] = {0.0, 0.0, 0.0};
    for (long long q = cf_ptr[c]; q < cf_ptr[c + 1]; ++q) {
      const int fe = cf_face[q];
      const int f = fe >> 1;
      const double sg = (fe & 1) ? -1.0 : 1.0;
      const long long lo = f_lo[f], hi = f_hi[f];
      const double wf = 0.5 * U[f];
      const double kd = aol[f] * visc;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double vl = vc[d * ncx + lo], vh = vc[d * ncx + hi];
        cv[d] += sg * (vl * wf + vh * wf);
        df[d] += sg * (kd * (vh - vl));
      }
    }
    const double vol = volci[c];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double conv = vol * cv[d], diff = vol * df[d];
      const double v = vc[d * ncx + c];
      if (mode == 0) {
        out0[d * nc + c] = conv;
        out1[d * nc + c] = diff;
      } else if (mode == 1) {
        out0[d * nc + c] = (rou * v - c1 * conv) + c2 * diff;
      } else {
        double rr = ((res0[d * nc + c] - rou * v) - c1 * conv) + c2 * diff;
        if (fE) rr = rr + dt * fE[d * nc + c];
        out0[d * nc + c] = rr;
      }
    }
  }
}

__global__ void k_guess(long long ne, double* s, double* s_old, double* prev, double dt, double dt_old) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const double se = s[e], so = s_old[e];
    prev[e] = se;
    s[e] = se + ((se - so) * dt) / dt_old;
    s_old[e] = se;
  }
}

// ---------------------------------------------------------------------------
// immersed boundary
// ---------------------------------------------------------------------------
__device__ __forceinline__ double delta_h3(double r, double h) {
  // Roma-Peskin 3-point kernel, ib_immersed.py:12-19 (same operation order)
  const double a = fabs(r / h);
  if (a <= 0.5) {
    double t = 1.0 - (3.0 * a) * a;
    t = t < 0.0 ? 0.0 : t;
    return (1.0 + sqrt(t)) / (3.0 * h);
  }
  if (a <= 1.5) {
    const double b = 1.0 - a;
    double t = 1.0 - 3.0 * (b * b);
    t = t < 0.0 ? 0.0 : t;
    return ((5.0 - 3.0 * a) - sqrt(t)) / (6.0 * h);
  }
  return 0.0;
}

// one thread per (marker, offset); base index per marker from rint((x - pos_ref)/dx)
__global__ void k_ib_stencil(int M, const double* __restrict__ mk, double px, double py, double pz,
                             double dx, double hh, int nx, int ny, int nz, int* cell, double* w,
                             int* base, int* err) {
  const long long tot = (long long)M * 125;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / 125), o = (int)(t % 125);
    const double x = mk[3 * i], y = mk[3 * i + 1], z = mk[3 * i + 2];
    const double bx = rint((x - px) / dx), by = rint((y - py) / dx), bz = rint((z - pz) / dx);
    if (!(fabs(bx) < 1e9 && fabs(by) < 1e9 && fabs(bz) < 1e9)) {
      cell[t] = 0; w[t] = 0.0;
      if (o == 0) atomicExch(err, 1);
      continue;
    }
    const long long lx = (long long)bx, ly = (long long)by, lz = (long long)bz;
    if (o == 0) { base[3 * i] = (int)lx; base[3 * i + 1] = (int)ly; base[3 * i + 2] = (int)lz; }
    const long long ii = lx + (o / 25) - 2, jj = ly + ((o / 5) % 5) - 2, kk = lz + (o % 5) - 2;
    const bool inb = ii >= 0 && ii < nx && jj >= 0 && jj < ny && kk >= 0 && kk < nz;
    const double gx = (px + (double)ii * dx) - x;
    const double gy = (py + (double)jj * dx) - y;
    const double gz = (pz + (double)kk * dx) - z;
    const double ww = (delta_h3(gx, hh) * delta_h3(gy, hh)) * delta_h3(gz, hh);
    if (inb) {
      cell[t] = (int)((kk * ny + jj) * nx + ii);      // level-0 dense id
      w[t] = ww;
    } else {
      cell[t] = 0;
      w[t] = 0.0;
    }
  }
}

// u_L = sum vc[cell] * (w * hh^3)    (ib_immersed.py:87-93)
__global__ void k_ib_interp(int M, long long ncx, const int* __restrict__ cell, const double* __restrict__ w,
                            double hh3, const double* __restrict__ vc, double* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int o = 0; o < 125; ++o) {
      const long long t = (long long)i * 125 + o;
      const double ww = w[t] * hh3;
      const int c = cell[t];
      a0 += vc[c] * ww;
      a1 += vc[ncx + c] * ww;
      a2 += vc[2 * ncx + c] * ww;
    }
    out[3 * i] = a0; out[3 * i + 1] = a1; out[3 * i + 2] = a2;
  }
}

// d/dr of delta_h3(r, h): the Roma-Peskin kernel is continuously differentiable
// (the slope is -1/h^2 from both sides at |r| = h/2 and 0 at |r| = 3h/2)
__device__ __forceinline__ double ddelta_h3(double r, double h) {
  const double a = fabs(r / h);
  double da;
  if (a <= 0.5) {
    const double t = 1.0 - (3.0 * a) * a;           // > 0 for a <= 1/2
    da = -a / sqrt(t);
  } else if (a <= 1.5) {
    const double b = 1.0 - a;
    const double t = 1.0 - 3.0 * (b * b);           // >= 1/4 for 1/2 < a <= 3/2
    da = (-3.0 - 3.0 * b / sqrt(t)) / 6.0;
  } else {
    return 0.0;
  }
  return (r < 0.0 ? -da : da) / (h * h);
}

// Jacobian of the interpolation with respect to the marker positions:
// jac[9 m + 3 c + d] = d u_L[m, c] / d x_m[d] = -hh^3 sum_o vc_c[cell_o] dw_o/dg_d, the
// weight w_o = delta(gx) delta(gy) delta(gz) with g = node - marker (ib_immersed.py:63-93).
// One thread per marker over the 125 offsets of its stencil base.
__global__ void k_ib_interp_dx(int M, long long ncx, const double* __restrict__ mk, double px, double py,
                               double pz, double dx, double hh, double hh3, int nx, int ny, int nz,
                               const int* __restrict__ base, const double* __restrict__ vc, double* jac) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    const double x = mk[3 * i], y = mk[3 * i + 1], z = mk[3 * i + 2];
    const long long lx = base[3 * i], ly = base[3 * i + 1], lz = base[3 * i + 2];
    double J[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int o = 0; o < 125; ++o) {
      const long long ii = lx + (o / 25) - 2, jj = ly + ((o / 5) % 5) - 2, kk = lz + (o % 5) - 2;
      if (!(ii >= 0 && ii < nx && jj >= 0 && jj < ny && kk >= 0 && kk < nz)) continue;
      const double gx = (px + (double)ii * dx) - x;
      const double gy = (py + (double)jj * dx) - y;
      const double gz = (pz + (double)kk * dx) - z;
      const double fx = delta_h3(gx, hh), fy = delta_h3(gy, hh), fz = delta_h3(gz, hh);
      const double wx = -(ddelta_h3(gx, hh) * fy) * fz;
      const double wy = -(fx * ddelta_h3(gy, hh)) * fz;
      const double wz = -(fx * fy) * ddelta_h3(gz, hh);
      const long long c = (kk * ny + jj) * nx + ii;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double v = vc[d * ncx + c] * hh3;
        J[3 * d] += v * wx;
        J[3 * d + 1] += v * wy;
        J[3 * d + 2] += v * wz;
      }
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) jac[9 * i + q] = J[q];
  }
}

__global__ void k_ib_keys(long long tot, const int* __restrict__ cell, const double* __restrict__ w,
                          int* keys, int* vals) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    keys[t] = cell[t];
    vals[t] = (int)t;
  }
}

// Segmented sums over cell-sorted contributions, in original (marker, offset)
// order inside each segment -- the order np.bincount adds them.
__global__ void k_ib_segsum(long long tot, long long nc, const int* __restrict__ keys,
                            const int* __restrict__ vals, const double* __restrict__ w,
                            const double* __restrict__ ds3, const double* __restrict__ f,
                            double* out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int key = keys[t];
    if (t > 0 && keys[t - 1] == key) continue;
    if (key < 0 || key >= nc) continue;            // rejected contributions (sentinel key nc)
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (long long q = t; q < tot && keys[q] == key; ++q) {
      const int src = vals[q];
      const int i = src / 125;
      const double ww = w[src] * ds3[i];
      a0 += f[3 * i] * ww;
      a1 += f[3 * i + 1] * ww;
      a2 += f[3 * i + 2] * ww;
    }
    out[key] = a0;
    out[nc + key] = a1;
    out[2 * nc + key] = a2;
  }
}

// f_L = (vel - u_L)/dt ; fL += rou*f_L ; dL = f_L
__global__ void k_ib_force(int M, const double* __restrict__ vel, const double* __restrict__ uL, double dt,
                           double* dL) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 3 * M; q += gridDim.x * blockDim.x)
    dL[q] = (vel[q] - uL[q]) / dt;
}

// y = a * x  (the direct force mode's replacement, ib_driver_np.py:480-481)
__global__ void k_set_scaled(long long n, double* y, double a, const double* __restrict__ x) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    y[q] = a * x[q];
}

// trace of the marker coupling matrix: sum_i ds_i^3 sum_k w_ik^2 (times hh^3 on the host)
__global__ void __launch_bounds__(kThreads) k_ib_trace(long long tot, const double* __restrict__ w,
                                                       const double* __restrict__ ds3, double* partials,
                                                       CGState* st, double* out) {
  double v[1] = {0.0};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x)
    v[0] += (w[t] * w[t]) * ds3[t / 125];
  if (grid_sum<1>(v, partials, &st->counter)) *out = v[0];
}

__global__ void k_axpy_scaled(long long n, double* y, double a, const double* x) {
  // y = y + (a * x)  (ib_driver_np.py:522-525)
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    y[q] = y[q] + a * x[q];
}

// ---------------------------------------------------------------------------
// loads and diagnostics
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_loads(long long ncand, const int* __restrict__ cand,
                                                    long long nf, const int* __restrict__ fidx,
                                                    const double* __restrict__ cpos,
                                                    const double* __restrict__ volci,
                                                    const double* __restrict__ vc, long long ncx,
                                                    const double* __restrict__ fE, long long nc,
                                                    double cx, double cy, double cz, double radius,
                                                    double width, double* partials, CGState* st,
                                                    double* out) {
  double v[13];
#pragma unroll
  for (int q = 0; q < 13; ++q) v[q] = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncand;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = cand[t];
    const double px = cpos[3 * (long long)c], py = cpos[3 * (long long)c + 1], pz = cpos[3 * (long long)c + 2];
    const double ddx = px - cx, ddy = py - cy, ddz = pz - cz;
    const double dist = sqrt((ddx * ddx + ddy * ddy) + ddz * ddz);
    double ind = (radius + 0.5 * width - dist) / width;
    ind = ind < 0.0 ? 0.0 : (ind > 1.0 ? 1.0 : ind);
    const double wv = ind * (1.0 / volci[c]);
    const double ux = vc[c], uy = vc[ncx + c], uz = vc[2 * ncx + c];
    v[6] += ux * wv; v[7] += uy * wv; v[8] += uz * wv;
    v[9] += (py * uz - pz * uy) * wv;
    v[10] += (pz * ux - px * uz) * wv;
    v[11] += (px * uy - py * ux) * wv;
    v[12] += wv;
  }
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nf;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = fidx[t];
    const double px = cpos[3 * (long long)c], py = cpos[3 * (long long)c + 1], pz = cpos[3 * (long long)c + 2];
    const double vol = 1.0 / volci[c];
    const double fx = fE[c], fy = fE[nc + c], fz = fE[2 * nc + c];
    v[0] += fx * vol; v[1] += fy * vol; v[2] += fz * vol;
    v[3] += (py * fz - pz * fy) * vol;
    v[4] += (pz * fx - px * fz) * vol;
    v[5] += (px * fy - py * fx) * vol;
  }
  if (grid_sum<13>(v, partials, &st->counter) && threadIdx.x == 0)
    for (int q = 0; q < 13; ++q) out[q] = v[q];
}

__global__ void __launch_bounds__(kThreads) k_diag(long long nc, long long ncx, const double* __restrict__ vc,
                                                   const long long* __restrict__ cf_ptr,
                                                   const int* __restrict__ cf_face,
                                                   const double* __restrict__ volci,
                                                   const double* __restrict__ U, double* partials,
                                                   CGState* st, double* out) {
  // max speed and max |vol * cdiv(U)| as sums of ... use max via separate slots
  __shared__ double sh[2][kThreads / 32];
  double smax = 0.0, dmax = 0.0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc;
       c += (long long)gridDim.x * blockDim.x) {
    if (volci[c] == 0.0) continue;
    const double a = vc[c], b = vc[ncx + c], d = vc[2 * ncx + c];
    const double sp = sqrt((a * a + b * b) + d * d);
    smax = fmax(smax, sp);
    double dv = 0.0;
    for (long long q = cf_ptr[c]; q < cf_ptr[c + 1]; ++q) {
      const int fe = cf_face[q];
      dv += ((fe & 1) ? -1.0 : 1.0) * U[fe >> 1];
    }
    dmax = fmax(dmax, fabs(volci[c] * dv));
  }
  for (int o = 16; o > 0; o >>= 1) {
    smax = fmax(smax, __shfl_down_sync(0xffffffffu, smax, o));
    dmax = fmax(dmax, __shfl_down_sync(0xffffffffu, dmax, o));
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sh[0][wid] = smax; sh[1][wid] = dmax; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) { smax = fmax(smax, sh[0][q]); dmax = fmax(dmax, sh[1][q]); }
    partials[blockIdx.x] = smax;
    partials[kPartStride + blockIdx.x] = dmax;
    __threadfence();
    unsigned int t = atomicAdd(&st->counter, 1u);
    if (t == gridDim.x - 1) {
      __threadfence();
      double a = 0.0, b = 0.0;
      for (int q = 0; q < (int)gridDim.x; ++q) {
        a = fmax(a, ((volatile double*)partials)[q]);
        b = fmax(b, ((volatile double*)partials)[kPartStride + q]);
      }
      out[0] = a; out[1] = b;
      st->counter = 0u;
    }
  }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
size_t table_elem(int t) {
  switch (t) {
    case PYIB_T_PREC: case PYIB_T_INLET_VAL: case PYIB_T_CURL_VAL: case PYIB_T_ROT_VAL:
    case PYIB_T_P_VAL3: case PYIB_T_I_VAL3: case PYIB_T_F_AOL: case PYIB_T_VOLCI:
    case PYIB_T_BF_AF: case PYIB_T_PA_VAL: case PYIB_T_PV_VAL: case PYIB_T_PR_VAL:
    case PYIB_T_LC_CPOS: case PYIB_T_PREC_REG:
      return 8;
    case PYIB_T_CURL_PTR: case PYIB_T_ROT_PTR: case PYIB_T_P_PTR: case PYIB_T_I_PTR:
    case PYIB_T_CF_PTR: case PYIB_T_PA_PTR: case PYIB_T_PV_PTR: case PYIB_T_PR_PTR:
      return 8;
    default:
      return 4;
  }
}

template <typename T>
T* tp(pyib_ctx* c, int t) { return (T*)c->tab[t].ptr; }

int alloc(pyib_ctx* ctx, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  CK(cudaMalloc(p, bytes));
  CK(cudaMemsetAsync(*p, 0, bytes, ctx->stream));
  return PYIB_OK;
}

int check_dev_err(pyib_ctx* ctx) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, ctx->dev_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (h) {
    CK(cudaMemsetAsync(ctx->dev_err, 0, sizeof(int), ctx->stream));
    return set_err(ctx, PYIB_E_DEVICE, "kernel-side check failed (code %d)", h);
  }
  return PYIB_OK;
}

bool tables_ready(pyib_ctx* c) {
  const int need[] = {PYIB_T_PREC, PYIB_T_PREC_BITS, PYIB_T_PREC_REG, PYIB_T_CURL_PTR, PYIB_T_ROT_PTR, PYIB_T_P_PTR, PYIB_T_I_PTR,
                      PYIB_T_CF_PTR, PYIB_T_F_LO, PYIB_T_F_HI, PYIB_T_F_AOL, PYIB_T_VOLCI, PYIB_T_PR_BITS};
  for (int t : need)
    if (!c->tab[t].ptr) return false;
  return true;
}

long long ncx_of(pyib_ctx* c) { return c->lay.ncell + c->lay.nbface; }

// ---- operators -------------------------------------------------------------
int op_curl(pyib_ctx* ctx, const double* s, double* U) {
  k_csr<<<grid_for(ctx->lay.nface), kThreads, 0, ctx->stream>>>(
      ctx->lay.nface, tp<long long>(ctx, PYIB_T_CURL_PTR), tp<int>(ctx, PYIB_T_CURL_COL),
      tp<double>(ctx, PYIB_T_CURL_VAL), s, U);
  CKL();
  return PYIB_OK;
}

int op_rot(pyib_ctx* ctx, const double* F, double* e) {
  k_csr<<<grid_for(ctx->lay.nedge), kThreads, 0, ctx->stream>>>(
      ctx->lay.nedge, tp<long long>(ctx, PYIB_T_ROT_PTR), tp<int>(ctx, PYIB_T_ROT_COL),
      tp<double>(ctx, PYIB_T_ROT_VAL), F, e);
  CKL();
  return PYIB_OK;
}

int op_interp(pyib_ctx* ctx, const double* U, double* vc, long long stride) {
  k_csr_to3<<<grid_for(ctx->lay.ncell), kThreads, 0, ctx->stream>>>(
      ctx->lay.ncell, stride, tp<long long>(ctx, PYIB_T_P_PTR), tp<int>(ctx, PYIB_T_P_COL),
      tp<double>(ctx, PYIB_T_P_VAL3), U, vc);
  CKL();
  return PYIB_OK;
}

int op_integr(pyib_ctx* ctx, const double* vc, long long stride, double* F) {
  k_csr_from3<<<grid_for(ctx->lay.nface), kThreads, 0, ctx->stream>>>(
      ctx->lay.nface, stride, tp<long long>(ctx, PYIB_T_I_PTR), tp<int>(ctx, PYIB_T_I_COL),
      tp<double>(ctx, PYIB_T_I_VAL3), vc, F);
  CKL();
  return PYIB_OK;
}

int op_calc_vel(pyib_ctx* ctx) {
  if (ctx->n_inlet > 0) {
    k_set_idx<<<grid_for(ctx->n_inlet), kThreads, 0, ctx->stream>>>(
        ctx->n_inlet, tp<int>(ctx, PYIB_T_INLET_IDX), tp<double>(ctx, PYIB_T_INLET_VAL), ctx->s);
    CKL();
  }
  RET(op_curl(ctx, ctx->s, ctx->U));
  const long long ncx = ncx_of(ctx);
  RET(op_interp(ctx, ctx->U, ctx->vc, ncx));
  if (ctx->n_bf > 0) {
    k_ghost<<<grid_for(ctx->n_bf), kThreads, 0, ctx->stream>>>(
        ctx->n_bf, ncx, ctx->lay.ncell, tp<int>(ctx, PYIB_T_BF_FACE), tp<int>(ctx, PYIB_T_BF_CELL),
        tp<int>(ctx, PYIB_T_BF_INFO), tp<double>(ctx, PYIB_T_BF_AF), ctx->U, ctx->vc);
    CKL();
  }
  return PYIB_OK;
}

int op_convdiff(pyib_ctx* ctx, int mode, double c1, double c2, double dt, const double* res0,
                const double* fE, double* out0, double* out1) {
  k_convdiff<<<grid_for(ctx->lay.ncell), kThreads, 0, ctx->stream>>>(
      ctx->lay.ncell, ncx_of(ctx), tp<long long>(ctx, PYIB_T_CF_PTR), tp<int>(ctx, PYIB_T_CF_FACE),
      tp<int>(ctx, PYIB_T_F_LO), tp<int>(ctx, PYIB_T_F_HI), tp<double>(ctx, PYIB_T_F_AOL),
      tp<double>(ctx, PYIB_T_VOLCI), ctx->U, ctx->vc, ctx->prm.visc, mode, ctx->prm.rou, c1, c2, dt,
      res0, fE, out0, out1);
  CKL();
  return PYIB_OK;
}

// ---- matvec ---------------------------------------------------------------
template <typename T>
int launch_matvec_t(pyib_ctx* ctx, const T* in, T* out, T* vcm, T* vq, const T* pdot, int alpd,
                    int do_dot, const T* pa_val, const T* pv_val, const T* pr_val) {
  const Meta& m = sizeof(T) == 4 ? ctx->meta32 : ctx->meta;
  const long long nc = ctx->lay.ncell;
  const dim3 blk(TX, TY, 1), gA(m.gxA, m.gyA, m.gzA), gV(m.gxV, m.gyA, m.gzA), gR(m.gxR, m.gyR, m.gzR);
  if (alpd && m.av && !ctx->flags_ready) return set_err(ctx, PYIB_E_STATE, "fused A+V kernel without its cell flags");
  if (!(alpd && m.av)) {
    k_mvA<T><<<gA, blk, 0, ctx->stream>>>(m, in, vcm, nullptr, nullptr, nullptr, nullptr, pa_val, ctx->nA,
                                          ctx->st);
    CKL();
  }
  if (ctx->nA > 0) {
    k_patchA<T><<<patch_grid(3 * ctx->nA), kThreads, 0, ctx->stream>>>(
        ctx->nA, tp<int>(ctx, PYIB_T_PA_IDS), tp<long long>(ctx, PYIB_T_PA_PTR), tp<int>(ctx, PYIB_T_PA_COL),
        pa_val, in, vcm, nc, ctx->st);
    CKL();
  }
  const T* vsrc = vcm;
  if (alpd && m.av) {
    // exact vc rows (k_patchA, above) first, then vq = V P C p in one pass, then the
    // exact vq rows
    k_mvAV<T><<<gA, blk, 0, ctx->stream>>>(m, in, vcm, vq, ctx->f_flags, ctx->st);
    CKL();
    if (ctx->nV > 0) {
      k_patchV<T><<<patch_grid(ctx->nV), kThreads, 0, ctx->stream>>>(
          ctx->nV, tp<int>(ctx, PYIB_T_PV_IDS), tp<long long>(ctx, PYIB_T_PV_PTR), tp<int>(ctx, PYIB_T_PV_COL),
          pv_val, vcm, vq, nc, ctx->st);
      CKL();
    }
    vsrc = vq;
  } else if (alpd) {
    k_mvV<T><<<gV, blk, 0, ctx->stream>>>(m, vcm, vq, ctx->st);
    CKL();
    if (ctx->nV > 0) {
      k_patchV<T><<<patch_grid(ctx->nV), kThreads, 0, ctx->stream>>>(
          ctx->nV, tp<int>(ctx, PYIB_T_PV_IDS), tp<long long>(ctx, PYIB_T_PV_PTR), tp<int>(ctx, PYIB_T_PV_COL),
          pv_val, vcm, vq, nc, ctx->st);
      CKL();
    }
    vsrc = vq;
  }
  k_mvRI<T><<<gR, blk, 0, ctx->stream>>>(m, vsrc, out, pdot, tp<unsigned int>(ctx, PYIB_T_PR_BITS),
                                          ctx->partials, ctx->st, do_dot);
  CKL();
  k_patchRI<T><<<patch_grid(ctx->nR), kThreads, 0, ctx->stream>>>(
      ctx->nR, tp<int>(ctx, PYIB_T_PR_IDS), tp<long long>(ctx, PYIB_T_PR_PTR), tp<int>(ctx, PYIB_T_PR_COL),
      pr_val, vsrc, out, pdot, ctx->partials, m.nplanes, ctx->st, do_dot);
  CKL();
  return PYIB_OK;
}

int launch_matvec(pyib_ctx* ctx, const double* in, double* out, int alpd, int do_dot) {
  return launch_matvec_t<double>(ctx, in, out, ctx->vcm, ctx->vq, ctx->p, alpd, do_dot,
                                 tp<double>(ctx, PYIB_T_PA_VAL), tp<double>(ctx, PYIB_T_PV_VAL),
                                 tp<double>(ctx, PYIB_T_PR_VAL));
}

// Flags and lists of the fused matvec, from the patch tables (once per table upload):
// irrA / irrV = cells with exact vc / vq rows, needR = cells whose vq an exact w row
// reads, and the list of regular cells whose template vc an exact vq row reads.
int prepare_flags(pyib_ctx* ctx) {
  if (ctx->flags_ready) return PYIB_OK;
  const long long nc = ctx->lay.ncell, words = (nc + 31) / 32;
  unsigned int** bits[] = {&ctx->f_irrA, &ctx->f_irrV, &ctx->f_needR};
  for (unsigned int** b : bits) {
    if (*b) { CK(cudaFree(*b)); *b = nullptr; }
    RET(alloc(ctx, (void**)b, words * sizeof(unsigned int)));
  }
  if (ctx->f_list) { CK(cudaFree(ctx->f_list)); ctx->f_list = nullptr; }
  if (ctx->nA > 0) {
    k_mark_cells<<<grid_for(ctx->nA), kThreads, 0, ctx->stream>>>(ctx->nA, tp<int>(ctx, PYIB_T_PA_IDS), nc,
                                                                    ctx->f_irrA);
    CKL();
  }
  if (ctx->nV > 0) {
    k_mark_cells<<<grid_for(ctx->nV), kThreads, 0, ctx->stream>>>(ctx->nV, tp<int>(ctx, PYIB_T_PV_IDS), nc,
                                                                    ctx->f_irrV);
    CKL();
  }
  if (ctx->nR > 0) {
    const long long nnz = (long long)(ctx->tab[PYIB_T_PR_COL].bytes / sizeof(int));
    k_mark_cells<<<grid_for(nnz), kThreads, 0, ctx->stream>>>(nnz, tp<int>(ctx, PYIB_T_PR_COL), nc, ctx->f_needR);
    CKL();
  }
  if (ctx->f_flags) { CK(cudaFree(ctx->f_flags)); ctx->f_flags = nullptr; }
  RET(alloc(ctx, (void**)&ctx->f_flags, nc));
  k_cell_flags<<<grid_for(nc), kThreads, 0, ctx->stream>>>(nc, ctx->f_irrA, ctx->f_irrV, ctx->f_needR,
                                                           ctx->f_flags);
  CKL();
  // cells read by the exact V rows (their columns and the rows' own cells), minus the
  // cells with exact vc: a host pass over the column list
  std::vector<int> cols;
  if (ctx->nV > 0) {
    const size_t nnz = ctx->tab[PYIB_T_PV_COL].bytes / sizeof(int);
    cols.resize(nnz + ctx->nV);
    CK(cudaMemcpyAsync(cols.data(), tp<int>(ctx, PYIB_T_PV_COL), nnz * sizeof(int), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaMemcpyAsync(cols.data() + nnz, tp<int>(ctx, PYIB_T_PV_IDS), ctx->nV * sizeof(int),
                       cudaMemcpyDeviceToHost, ctx->stream));
  }
  std::vector<unsigned int> irrA(words);
  CK(cudaMemcpyAsync(irrA.data(), ctx->f_irrA, words * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<char> want(nc, 0);
  for (int c : cols)
    if (c >= 0 && c < nc && !((irrA[c >> 5] >> (c & 31)) & 1u)) want[c] = 1;
  std::vector<int> list;
  for (long long c = 0; c < nc; ++c)
    if (want[c]) list.push_back((int)c);
  ctx->n_list = (long long)list.size();
  RET(alloc(ctx, (void**)&ctx->f_list, std::max<size_t>(1, list.size()) * sizeof(int)));
  if (!list.empty()) {
    CK(cudaMemcpyAsync(ctx->f_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    k_flag_list<<<grid_for(ctx->n_list), kThreads, 0, ctx->stream>>>(ctx->n_list, ctx->f_list, nc, kFlagStoreVc,
                                                                     ctx->f_flags);
    CKL();
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->flags_ready = true;
  return PYIB_OK;
}

// prepare_flags plus the single-pass kernel's reduction slots and shared memory
int prepare_fused(pyib_ctx* ctx) {
  if (ctx->fused_ready) return PYIB_OK;
  RET(prepare_flags(ctx));
  if ((long long)ctx->meta.nplanesF + patch_grid(ctx->nR) > kPartStride)
    return set_err(ctx, PYIB_E_ARG, "too many reduction slots for the fused matvec");
  CK(cudaFuncSetAttribute(k_mvF, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedSmemBytes));
  ctx->fused_ready = true;
  return PYIB_OK;
}

// The float64 matvec as one pass: exact vc / vq rows first, then k_mvF, then the exact
// w rows with the final dot (alpha = eta / p.w when do_dot).
int launch_matvec_fused(pyib_ctx* ctx, const double* in, double* out, int do_dot) {
  RET(prepare_fused(ctx));
  const Meta& m = ctx->meta;
  const long long nc = ctx->lay.ncell;
  if (ctx->nA > 0) {
    k_patchA<double><<<patch_grid(3 * ctx->nA), kThreads, 0, ctx->stream>>>(
        ctx->nA, tp<int>(ctx, PYIB_T_PA_IDS), tp<long long>(ctx, PYIB_T_PA_PTR), tp<int>(ctx, PYIB_T_PA_COL),
        tp<double>(ctx, PYIB_T_PA_VAL), in, ctx->vcm, nc, ctx->st);
    CKL();
  }
  if (ctx->n_list > 0) {
    k_vc_list<<<patch_grid(ctx->n_list), kThreads, 0, ctx->stream>>>(m, ctx->n_list, ctx->f_list, in, ctx->vcm,
                                                                      ctx->st);
    CKL();
  }
  if (ctx->nV > 0) {
    k_patchV<double><<<patch_grid(ctx->nV), kThreads, 0, ctx->stream>>>(
        ctx->nV, tp<int>(ctx, PYIB_T_PV_IDS), tp<long long>(ctx, PYIB_T_PV_PTR), tp<int>(ctx, PYIB_T_PV_COL),
        tp<double>(ctx, PYIB_T_PV_VAL), ctx->vcm, ctx->vq, nc, ctx->st);
    CKL();
  }
  const FusedTabs tb{ctx->f_irrA, ctx->f_irrV, ctx->f_needR, tp<unsigned int>(ctx, PYIB_T_PR_BITS),
                     ctx->f_flags};
  k_mvF<<<dim3(m.gxF, m.gyF, m.gzF), dim3(FX, FY, 1), kFusedSmemBytes, ctx->stream>>>(m, in, out, ctx->vcm, ctx->vq, tb,
                                                                       ctx->partials, ctx->st, do_dot);
  CKL();
  k_patchRI<double><<<patch_grid(ctx->nR), kThreads, 0, ctx->stream>>>(
      ctx->nR, tp<int>(ctx, PYIB_T_PR_IDS), tp<long long>(ctx, PYIB_T_PR_PTR), tp<int>(ctx, PYIB_T_PR_COL),
      tp<double>(ctx, PYIB_T_PR_VAL), ctx->vq, out, in, ctx->partials, m.nplanesF, ctx->st, do_dot);
  CKL();
  return PYIB_OK;
}

// Depth of the fused matvec's z chunks, by timing 4, 8, 16 and 32 node planes.
int tune_fused(pyib_ctx* ctx) {
  if (ctx->tunedF) return PYIB_OK;
  RET(prepare_fused(ctx));
  CGState h{};
  CK(cudaMemcpyAsync(&h, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CGState t = h;
  t.rou = 1.0;
  t.kfac = 1e-3;
  t.done = 0;
  t.counter = 0u;
  CK(cudaMemcpyAsync(ctx->st, &t, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  const int depths[4] = {4, 8, 16, 32};
  int bestZ = 16;
  double best = 1e30;
  for (int a = 0; a < 4; ++a) {
    set_grids_fused(ctx->meta, depths[a]);
    RET(launch_matvec_fused(ctx, ctx->work_e, ctx->work_e2, 0));
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int q = 0; q < 3; ++q) RET(launch_matvec_fused(ctx, ctx->work_e, ctx->work_e2, 0));
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (ms < best) {
      best = ms;
      bestZ = depths[a];
    }
  }
  set_grids_fused(ctx->meta, bestZ);
  ctx->tunedF = true;
  ctx->cg_graph_check = -1;
  CK(cudaMemcpyAsync(ctx->st, &h, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

constexpr int kTuneReps = 4;   // products per timing of one tuner configuration

// Matvec forms the autotuners try: kernels A and V as two kernels (0) and fused (1).
// PYIB_MATVEC_AV=0 or =1 (read at context creation) pins one of them.
int av_lo(const pyib_ctx* ctx) { return ctx->av_pin == 1 ? 1 : 0; }
int av_hi(const pyib_ctx* ctx) { return ctx->av_pin == 0 ? 0 : 1; }

// Autotuner: time the float64 matvec for every pair of z-chunk depths (cells, nodes),
// with kernels A and V apart and fused, and keep the fastest.  Runs once per context, before any CG graph is captured.
int tune_matvec(pyib_ctx* ctx) {
  if (ctx->tuned) return PYIB_OK;
  CGState h{};
  CK(cudaMemcpyAsync(&h, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CGState t = h;
  t.rou = 1.0;
  t.kfac = 1e-3;
  t.done = 0;
  t.counter = 0u;
  CK(cudaMemcpyAsync(ctx->st, &t, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  const int depths[5] = {1, 2, 4, 8, 16};
  RET(prepare_flags(ctx));
  const Meta base = ctx->meta;
  int bestA = base.kz, bestR = base.kzR, bestAV = 0;
  double best = 1e30;
  for (int av = av_lo(ctx); av <= av_hi(ctx); ++av) {
    for (int a = 0; a < 5; ++a) {
      for (int b = 0; b < 5; ++b) {
        Meta m2 = base;
        set_grids(m2, depths[a], depths[b]);
        m2.av = av;
        if ((long long)m2.gxR * m2.gyR * m2.gzR > kPartStride) continue;
        ctx->meta = m2;
        RET(launch_matvec(ctx, ctx->work_e, ctx->work_e2, 1, 0));
        // the better of two timings of kTuneReps products: one noisy sample must not
        // decide the tiles of every later solve
        float ms = 1e30f;
        for (int t = 0; t < 2; ++t) {
          CK(cudaEventRecord(ctx->ev0, ctx->stream));
          for (int q = 0; q < kTuneReps; ++q) RET(launch_matvec(ctx, ctx->work_e, ctx->work_e2, 1, 0));
          CK(cudaEventRecord(ctx->ev1, ctx->stream));
          CK(cudaEventSynchronize(ctx->ev1));
          float mt = 0.f;
          CK(cudaEventElapsedTime(&mt, ctx->ev0, ctx->ev1));
          ms = std::min(ms, mt);
        }
        if (ms < best) {
          best = ms;
          bestA = depths[a];
          bestR = depths[b];
          bestAV = av;
        }
      }
    }
  }
  ctx->meta = base;
  set_grids(ctx->meta, bestA, bestR);
  ctx->meta.av = bestAV;
  ctx->tune_ms = best / kTuneReps;
  ctx->tuned = true;
  ctx->cg_graph_check = -1;
  ctx->mix_graph_check = -1;
  CK(cudaMemcpyAsync(ctx->st, &h, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

// The same search for the float32 matvec of the mixed solver: its kernels wait on
// load latency differently, so they get their own depths (meta32).  The dot's
// partials are indexed by plane, not by chunk, so the depths do not change results.
int tune_matvec32(pyib_ctx* ctx) {
  if (ctx->tuned32) return PYIB_OK;
  CGState h{};
  CK(cudaMemcpyAsync(&h, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CGState t = h;
  t.rou = 1.0;
  t.kfac = 1e-3;
  t.done = 0;
  t.counter = 0u;
  CK(cudaMemcpyAsync(ctx->st, &t, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  const long long ne = ctx->lay.nedge;
  CK(cudaMemsetAsync(ctx->p32, 0, ne * sizeof(float), ctx->stream));
  const int depths[5] = {1, 2, 4, 8, 16};
  RET(prepare_flags(ctx));
  const Meta base = ctx->meta;
  int bestA = base.kz, bestR = base.kzR, bestAV = 0;
  double best = 1e30;
  for (int av = av_lo(ctx); av <= av_hi(ctx); ++av) {
    for (int a = 0; a < 5; ++a) {
      for (int b = 0; b < 5; ++b) {
        Meta m2 = base;
        set_grids(m2, depths[a], depths[b]);
        m2.av = av;
        if ((long long)m2.gxR * m2.gyR * m2.gzR > kPartStride) continue;
        ctx->meta32 = m2;
        auto once = [&]() {
          return launch_matvec_t<float>(ctx, ctx->p32, ctx->w32, ctx->vcm32, ctx->vq32, ctx->p32, 1, 0,
                                        ctx->pa_val32, ctx->pv_val32, ctx->pr_val32);
        };
        RET(once());
        float ms = 1e30f;
        for (int t = 0; t < 2; ++t) {
          CK(cudaEventRecord(ctx->ev0, ctx->stream));
          for (int q = 0; q < kTuneReps; ++q) RET(once());
          CK(cudaEventRecord(ctx->ev1, ctx->stream));
          CK(cudaEventSynchronize(ctx->ev1));
          float mt = 0.f;
          CK(cudaEventElapsedTime(&mt, ctx->ev0, ctx->ev1));
          ms = std::min(ms, mt);
        }
        if (ms < best) {
          best = ms;
          bestA = depths[a];
          bestR = depths[b];
          bestAV = av;
        }
      }
    }
  }
  ctx->meta32 = base;
  set_grids(ctx->meta32, bestA, bestR);
  ctx->meta32.av = bestAV;
  ctx->tuned32 = true;
  ctx->mix_graph_check = -1;
  CK(cudaMemcpyAsync(ctx->st, &h, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int set_state_solver(pyib_ctx* ctx, double dt, int alpd) {
  CGState h{};
  CK(cudaMemcpyAsync(&h, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  h.tol1 = ctx->prm.tol1;
  h.tol2 = ctx->prm.tol2;
  h.rou = ctx->prm.rou;
  h.kfac = 0.5 * dt * ctx->prm.visc;
  h.check = ctx->prm.check;
  h.cg_max = ctx->prm.cg_max;
  h.alpd = alpd;
  h.done = 0;
  h.stop = 0;
  h.counter = 0u;
  h.counter2 = 0u;
  CK(cudaMemcpyAsync(ctx->st, &h, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  return PYIB_OK;
}

int masked_matvec(pyib_ctx* ctx, const double* in, double* out, double dt, int alpd) {
  RET(set_state_solver(ctx, dt, alpd & 1));
  if (alpd & 2) {
    // the single-pass fused matvec (viscous block always on)
    if (!(alpd & 1)) return set_err(ctx, PYIB_E_ARG, "the fused matvec needs the viscous block (alpd 3)");
    if (!ctx->tunedF) set_grids_fused(ctx->meta, ctx->meta.kzF > 0 ? ctx->meta.kzF : 16);
    return launch_matvec_fused(ctx, in, out, 0);
  }
  if (alpd & 12) {
    // kernels A and V pinned: fused (4) or apart (8), viscous block on
    if (!(alpd & 1)) return set_err(ctx, PYIB_E_ARG, "a pinned A/V form needs the viscous block (alpd 5 or 9)");
    RET(prepare_flags(ctx));
    const int keep = ctx->meta.av;
    ctx->meta.av = (alpd & 4) ? 1 : 0;
    const int rc = launch_matvec(ctx, in, out, 1, 0);
    ctx->meta.av = keep;
    return rc;
  }
  RET(launch_matvec(ctx, in, out, alpd, 0));
  return PYIB_OK;
}

// one CG iteration (5 kernels)
int cg_iteration(pyib_ctx* ctx) {
  if (ctx->use_fused)
    RET(launch_matvec_fused(ctx, ctx->p, ctx->w, 1));
  else
    RET(launch_matvec(ctx, ctx->p, ctx->w, 1, 1));
  const long long ne = ctx->lay.nedge;
  const unsigned int* pb = tp<unsigned int>(ctx, PYIB_T_PREC_BITS);
  k_cg_update<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ctx->meta, ne, ctx->r, ctx->w, pb,
                                                          tp<double>(ctx, PYIB_T_PREC), ctx->partials,
                                                          ctx->st);
  CKL();
  k_cg_p<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ctx->meta, ne, ctx->r, pb, tp<double>(ctx, PYIB_T_PREC),
                                                     ctx->p, ctx->x, ctx->st);
  CKL();
  return PYIB_OK;
}

// kernel nodes of a captured graph (the launch count of one replay)
long long graph_kernels(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
  long long k = 0;
  for (size_t i = 0; i < n; ++i) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

int build_cg_graph(pyib_ctx* ctx) {
  if (ctx->cg_graph && ctx->cg_graph_check == ctx->prm.check) return PYIB_OK;
  if (ctx->cg_graph) {
    cudaGraphExecDestroy(ctx->cg_graph);
    ctx->cg_graph = nullptr;
  }
  cudaGraph_t g;
  const long long launched = ctx->launches;   // captured launches are counted per replay instead
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int rc = PYIB_OK;
  for (int q = 0; q < ctx->prm.check && rc == PYIB_OK; ++q) rc = cg_iteration(ctx);
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  ctx->launches = launched;
  if (rc != PYIB_OK) return rc;
  if (e != cudaSuccess) return set_err(ctx, PYIB_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  ctx->cg_graph_kernels = graph_kernels(g);
  e = cudaGraphInstantiate(&ctx->cg_graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_err(ctx, PYIB_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
  ctx->cg_graph_check = ctx->prm.check;
  return PYIB_OK;
}

// PCG from warm start s with right-hand side residual res_e (ib_driver_np.py:311-410),
// in three parts so that a batch can run the iterations of many cases together:
// solve_begin (tuning, state, k_cg_init; *iterate is false when the start already
// meets the test), the iteration chunks (this context's CG graph, or a batched one),
// and solve_end (true residual of the correction, s = x, statistics).
int solve_begin(pyib_ctx* ctx, double dt, bool own_graph, bool* iterate) {
  const long long ne = ctx->lay.nedge;
  const double* prec = tp<double>(ctx, PYIB_T_PREC);
  RET(tune_matvec(ctx));
  if (ctx->use_fused) RET(tune_fused(ctx));
  RET(set_state_solver(ctx, dt, 1));
  if (own_graph) RET(build_cg_graph(ctx));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  k_cg_init<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->res_e, ctx->s, prec, ctx->x, ctx->r,
                                                        ctx->p, ctx->partials, ctx->st);
  CKL();
  CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *iterate = !(ctx->st_host->eta < ctx->st_host->thresh);
  return PYIB_OK;
}

int solve_end(pyib_ctx* ctx, bool iterated, pyib_solve_stats* out) {
  const long long ne = ctx->lay.nedge;
  const double* prec = tp<double>(ctx, PYIB_T_PREC);
  int iters = 0;
  if (iterated) {
    if (!ctx->st_host->done) return set_err(ctx, PYIB_E_STATE, "CG loop did not terminate");
    iters = ctx->st_host->iters;
    // true residual of the correction x - s (ib_driver_np.py:404-410)
    k_sub<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->x, ctx->s, ctx->work_e2);
    CKL();
    {
      // the matvec kernels skip work while done is set; clear it for this product
      int zero = 0;
      CK(cudaMemcpyAsync(&ctx->st->done, &zero, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    }
    RET(launch_matvec(ctx, ctx->work_e2, ctx->w, 1, 0));
    k_cg_true<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->res_e, ctx->w, prec, 1, ctx->partials,
                                                          ctx->st);
    CKL();
  } else {
    k_cg_true<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->res_e, nullptr, prec, 0, ctx->partials,
                                                          ctx->st);
    CKL();
  }
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(ctx->s, ctx->x, ne * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->cg_seconds += ms * 1e-3;
  ctx->cg_iters += iters;
  const CGState& h = *ctx->st_host;
  const double eta_f = h.true_eta, l2_f = h.true_l2, l2_0 = h.l2_0, thr = h.thresh;
  const bool finite = std::isfinite(eta_f) && std::isfinite(l2_f) && std::isfinite(l2_0) &&
                      std::isfinite(thr) && eta_f >= 0 && l2_f >= 0 && l2_0 >= 0 && thr >= 0;
  pyib_solve_stats s{};
  s.iterations = iters;
  s.rel_residual = finite && l2_0 > 0 ? std::sqrt(l2_f / l2_0) : (finite && l2_f == 0 ? 0.0 : INFINITY);
  s.tol_ratio = finite && thr > 0 ? std::sqrt(eta_f / thr) : (finite && eta_f == 0 ? 0.0 : INFINITY);
  s.converged = finite && eta_f <= thr;
  s.eta0 = h.eta;
  s.threshold = thr;
  if (out) *out = s;
  if (ctx->prm.strict && !s.converged)
    return set_err(ctx, PYIB_E_NOCONV,
                   "Helmholtz CG did not converge: iterations=%d/%d, true_relative_residual=%.6e, "
                   "mixed_tolerance_ratio=%.6e",
                   iters, ctx->prm.cg_max, s.rel_residual, s.tol_ratio);
  return PYIB_OK;
}

// chunks of `check` iterations bounded by cg_max: the most a solve can replay
long long max_cg_chunks(const pyib_ctx* ctx) {
  return (ctx->prm.cg_max + ctx->prm.check - 1) / ctx->prm.check + 1;
}

int helm_solve(pyib_ctx* ctx, double dt, pyib_solve_stats* out) {
  bool iterate = false;
  RET(solve_begin(ctx, dt, true, &iterate));
  if (iterate) {
    for (long long q = 0; q < max_cg_chunks(ctx); ++q) {
      CK(cudaGraphLaunch(ctx->cg_graph, ctx->stream));
      ctx->launches += ctx->cg_graph_kernels;
      CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      if (ctx->st_host->done) break;
    }
  }
  return solve_end(ctx, iterate, out);
}

// ---- mixed precision --------------------------------------------------------
int set_state_raw(pyib_ctx* ctx, double rou, double kfac) {
  CGState h{};
  CK(cudaMemcpyAsync(&h, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  h.rou = rou;
  h.kfac = kfac;
  h.done = 0;
  h.counter = 0u;
  CK(cudaMemcpyAsync(ctx->st, &h, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  return PYIB_OK;
}

int ensure_mixed(pyib_ctx* ctx) {
  if (ctx->r32) return PYIB_OK;
  const long long ne = ctx->lay.nedge, nc = ctx->lay.ncell;
  float** ef[] = {&ctx->r32, &ctx->p32, &ctx->w32, &ctx->x32, &ctx->prec32};
  for (float** f : ef) RET(alloc(ctx, (void**)f, ne * sizeof(float)));
  RET(alloc(ctx, (void**)&ctx->vcm32, 3 * nc * sizeof(float)));
  RET(alloc(ctx, (void**)&ctx->vq32, 3 * nc * sizeof(float)));
  RET(alloc(ctx, (void**)&ctx->diag1, ne * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->diag2, ne * sizeof(double)));
  const int tabs[3] = {PYIB_T_PA_VAL, PYIB_T_PV_VAL, PYIB_T_PR_VAL};
  float** outs[3] = {&ctx->pa_val32, &ctx->pv_val32, &ctx->pr_val32};
  for (int q = 0; q < 3; ++q) {
    const long long n = (long long)(ctx->tab[tabs[q]].bytes / 8);
    RET(alloc(ctx, (void**)outs[q], (n > 0 ? n : 1) * sizeof(float)));
    if (n > 0) {
      k_d2f<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, tp<double>(ctx, tabs[q]), *outs[q]);
      CKL();
    }
  }
  return PYIB_OK;
}

// diag(A) = rou*diag1 + kfac*diag2 by probing with one colour of edges at a time:
// same level and axis, index residues mod 5 (A couples edges at most 3 apart, so no
// two edges of one colour share a row entry).
int build_diag(pyib_ctx* ctx) {
  if (ctx->diag_ready) return PYIB_OK;
  const long long ne = ctx->lay.nedge;
  const int q = 5;
  double* probe = ctx->work_e;
  double* out = ctx->w;
  CK(cudaMemsetAsync(probe, 0, ne * sizeof(double), ctx->stream));
  for (int pass = 0; pass < 2; ++pass) {
    RET(set_state_raw(ctx, pass == 0 ? 1.0 : 0.0, pass == 0 ? 0.0 : 1.0));
    double* dst = pass == 0 ? ctx->diag1 : ctx->diag2;
    for (int L = 0; L < ctx->meta.nl; ++L) {
      const LevelMeta& l = ctx->meta.lv[L];
      for (int a = 0; a < 3; ++a) {
        const int dx = l.n[0] + (a != 0), dy = l.n[1] + (a != 1);
        const int cnt = (int)l.ecount[a];
        const long long base = l.ebase[a];
        const int g = grid_for(cnt);
        for (int ci = 0; ci < q; ++ci)
          for (int cj = 0; cj < q; ++cj)
            for (int ck = 0; ck < q; ++ck) {
              k_probe_set<<<g, kThreads, 0, ctx->stream>>>(cnt, 0, dx, dy, cnt, q, ci, cj, ck, probe + base, 0);
              CKL();
              RET(launch_matvec(ctx, probe, out, pass, 0));
              k_probe_get<<<g, kThreads, 0, ctx->stream>>>(base, dx, dy, cnt, q, ci, cj, ck, out, dst);
              CKL();
              k_probe_set<<<g, kThreads, 0, ctx->stream>>>(cnt, 0, dx, dy, cnt, q, ci, cj, ck, probe + base, 1);
              CKL();
            }
      }
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->diag_ready = true;
  return PYIB_OK;
}

int mix_iteration(pyib_ctx* ctx) {
  RET(launch_matvec_t<float>(ctx, ctx->p32, ctx->w32, ctx->vcm32, ctx->vq32, ctx->p32, 1, 1,
                             ctx->pa_val32, ctx->pv_val32, ctx->pr_val32));
  const long long ne = ctx->lay.nedge;
  k_cg_update32<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->x32, ctx->r32, ctx->p32, ctx->w32,
                                                            ctx->prec32, ctx->partials, ctx->st);
  CKL();
  k_cg_p32<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->r32, ctx->prec32, ctx->p32, ctx->st);
  CKL();
  return PYIB_OK;
}

int build_mix_graph(pyib_ctx* ctx) {
  if (ctx->mix_graph && ctx->mix_graph_check == ctx->prm.check) return PYIB_OK;
  if (ctx->mix_graph) {
    cudaGraphExecDestroy(ctx->mix_graph);
    ctx->mix_graph = nullptr;
  }
  cudaGraph_t g;
  const long long launched = ctx->launches;   // captured launches are counted per replay instead
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int rc = PYIB_OK;
  for (int q = 0; q < ctx->prm.check && rc == PYIB_OK; ++q) rc = mix_iteration(ctx);
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  ctx->launches = launched;
  if (rc != PYIB_OK) return rc;
  if (e != cudaSuccess) return set_err(ctx, PYIB_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  ctx->mix_graph_kernels = graph_kernels(g);
  e = cudaGraphInstantiate(&ctx->mix_graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_err(ctx, PYIB_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
  ctx->mix_graph_check = ctx->prm.check;
  return PYIB_OK;
}

int clear_done(pyib_ctx* ctx) {
  int zero = 0;
  CK(cudaMemcpyAsync(&ctx->st->done, &zero, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  return PYIB_OK;
}

// State of one mixed-precision solve between its parts (mixed_begin, the float32
// iteration chunks, mixed_refine after each inner stop, mixed_end).
struct MixRun {
  double thresh = 0, l2_0 = 0, eta0 = 0, eta = 0, l2 = 0, eps2 = 0;
  int inner_total = 0, sweeps = 0, max_sweeps = 40;
};

int mixed_begin(pyib_ctx* ctx, double dt, bool own_graph, MixRun& mr, bool* iterate) {
  const long long ne = ctx->lay.nedge;
  const double* prec = tp<double>(ctx, PYIB_T_PREC);
  RET(tune_matvec(ctx));
  RET(ensure_mixed(ctx));
  RET(tune_matvec32(ctx));
  RET(build_diag(ctx));
  const double kfac = 0.5 * dt * ctx->prm.visc;
  if (ctx->diag_for_kfac != kfac || ctx->diag_for_rou != ctx->prm.rou) {
    k_dinv<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->diag1, ctx->diag2, prec, ctx->prm.rou, kfac,
                                                      ctx->prec32);
    CKL();
    ctx->diag_for_kfac = kfac;
    ctx->diag_for_rou = ctx->prm.rou;
  }
  RET(set_state_solver(ctx, dt, 1));
  if (own_graph) RET(build_mix_graph(ctx));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  k_cg_init<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->res_e, ctx->s, prec, ctx->x, ctx->r,
                                                        ctx->p, ctx->partials, ctx->st);
  CKL();
  CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  mr = MixRun{};
  mr.thresh = ctx->st_host->thresh;
  mr.l2_0 = ctx->st_host->l2_0;
  mr.eta0 = ctx->st_host->eta;
  mr.eta = mr.eta0;
  mr.l2 = mr.l2_0;
  mr.eps2 = ctx->prm.mixed_tol * ctx->prm.mixed_tol;
  mr.max_sweeps = ctx->prm.mixed_max_sweeps > 0 ? ctx->prm.mixed_max_sweeps : 40;
  // One float32 PCG (Jacobi on diag A) with reliable updates.  Whenever its residual
  // has dropped by mixed_tol since the last update, the float32 correction is folded
  // into x in float64 and r is recomputed in float64 (r -= A x32); the float32 CG then
  // continues from the new residual with the same search direction (no restart), and
  // the reference's float64 test on r decides when to stop.
  k_mix_start<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->r, ctx->prec32, ctx->r32, ctx->x32,
                                                          ctx->p32, mr.eps2, ctx->partials, ctx->st);
  CKL();
  *iterate = !(mr.eta < mr.thresh) && mr.sweeps < mr.max_sweeps;
  return PYIB_OK;
}

// After the float32 CG stopped (st_host read): x += x32, r -= A x32 in float64, the
// reference's test on r; unless it holds, the float32 CG continues from the new
// residual (*iterate stays true while sweeps remain).
int mixed_refine(pyib_ctx* ctx, MixRun& mr, bool* iterate) {
  const long long ne = ctx->lay.nedge;
  const double* prec = tp<double>(ctx, PYIB_T_PREC);
  double* d = ctx->p;                 // float64 copy of the float32 correction
  double* q = ctx->w;                 // A d
  mr.inner_total += ctx->st_host->iters;
  k_mix_widen<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->x32, d, prec);
  CKL();
  RET(clear_done(ctx));
  RET(launch_matvec(ctx, d, q, 1, 0));
  k_mix_fold<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, d, q, ctx->x, ctx->r, prec, ctx->partials, ctx->st);
  CKL();
  CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  mr.eta = ctx->st_host->true_eta;
  mr.l2 = ctx->st_host->true_l2;
  ++mr.sweeps;
  if (!std::isfinite(mr.eta) || mr.eta < mr.thresh) {
    *iterate = false;
    return PYIB_OK;
  }
  k_mix_reliable<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->r, ctx->prec32, ctx->r32, ctx->x32,
                                                             mr.eps2, ctx->partials, ctx->st);
  CKL();
  k_cg_p32<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->r32, ctx->prec32, ctx->p32, ctx->st);
  CKL();
  *iterate = mr.sweeps < mr.max_sweeps;
  return PYIB_OK;
}

int mixed_end(pyib_ctx* ctx, const MixRun& mr, pyib_solve_stats* out) {
  const long long ne = ctx->lay.nedge;
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaMemcpyAsync(ctx->s, ctx->x, ne * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->cg_seconds += ms * 1e-3;
  ctx->cg_iters += mr.inner_total;
  const double eta = mr.eta, l2 = mr.l2, l2_0 = mr.l2_0, thresh = mr.thresh;
  const bool finite = std::isfinite(eta) && std::isfinite(l2) && eta >= 0 && l2 >= 0;
  pyib_solve_stats st{};
  st.iterations = mr.inner_total;
  st.refinements = mr.sweeps;
  st.rel_residual = finite && l2_0 > 0 ? std::sqrt(l2 / l2_0) : (finite && l2 == 0 ? 0.0 : INFINITY);
  st.tol_ratio = finite && thresh > 0 ? std::sqrt(eta / thresh) : (finite && eta == 0 ? 0.0 : INFINITY);
  st.converged = finite && eta <= thresh;
  st.eta0 = mr.eta0;
  st.threshold = thresh;
  if (out) *out = st;
  if (ctx->prm.strict && !st.converged)
    return set_err(ctx, PYIB_E_NOCONV,
                   "mixed-precision Helmholtz solve did not converge: sweeps=%d, inner iterations=%d, "
                   "mixed_tolerance_ratio=%.6e",
                   mr.sweeps, mr.inner_total, st.tol_ratio);
  return PYIB_OK;
}

// Mixed precision: the float64 stopping test of helm_solve on the float64 residual,
// reached by one float32 PCG (Jacobi on diag(A)) with reliable float64 updates.
int helm_solve_mixed(pyib_ctx* ctx, double dt, pyib_solve_stats* out) {
  MixRun mr;
  bool iterate = false;
  RET(mixed_begin(ctx, dt, true, mr, &iterate));
  while (iterate) {
    for (long long c = 0; c < max_cg_chunks(ctx); ++c) {
      CK(cudaGraphLaunch(ctx->mix_graph, ctx->stream));
      ctx->launches += ctx->mix_graph_kernels;
      CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      if (ctx->st_host->done) break;
    }
    RET(mixed_refine(ctx, mr, &iterate));
  }
  return mixed_end(ctx, mr, out);
}

// ---- immersed boundary --------------------------------------------------
int ib_stencil(pyib_ctx* ctx) {
  if (ctx->M <= 0) return set_err(ctx, PYIB_E_STATE, "no markers");
  const long long tot = (long long)ctx->M * 125;
  k_ib_stencil<<<grid_for(tot), kThreads, 0, ctx->stream>>>(
      ctx->M, ctx->mk, ctx->pos_ref[0], ctx->pos_ref[1], ctx->pos_ref[2], ctx->dx, ctx->prm.hh,
      ctx->ib_n[0], ctx->ib_n[1], ctx->ib_n[2], ctx->ibcell, ctx->ibw, ctx->ibbase, ctx->dev_err);
  CKL();
  ctx->stencil_valid = true;
  return PYIB_OK;
}

int ib_interp(pyib_ctx* ctx, double* out) {
  k_ib_interp<<<grid_for(ctx->M), kThreads, 0, ctx->stream>>>(ctx->M, ncx_of(ctx), ctx->ibcell, ctx->ibw,
                                                              ctx->prm.hh3, ctx->vc, out);
  CKL();
  return PYIB_OK;
}

int ib_spread(pyib_ctx* ctx, const double* f, double* out) {
  const long long tot = (long long)ctx->M * 125, nc = ctx->lay.ncell;
  CK(cudaMemsetAsync(out, 0, 3 * nc * sizeof(double), ctx->stream));
  k_ib_keys<<<grid_for(tot), kThreads, 0, ctx->stream>>>(tot, ctx->ibcell, ctx->ibw, ctx->sort_keys_in,
                                                         ctx->sort_vals_in);
  CKL();
  int nbits = 1;
  while (nbits < 31 && (1LL << nbits) < ctx->lay.ncell) ++nbits;
  size_t tb = ctx->sort_tmp_bytes;
  CK(cub::DeviceRadixSort::SortPairs(ctx->sort_tmp, tb, ctx->sort_keys_in, ctx->sort_keys_out,
                                     ctx->sort_vals_in, ctx->sort_vals_out, (int)tot, 0, nbits,
                                     ctx->stream));
  k_ib_segsum<<<grid_for(tot), kThreads, 0, ctx->stream>>>(tot, nc, ctx->sort_keys_out, ctx->sort_vals_out,
                                                           ctx->ibw, ctx->ds, f, out);
  CKL();
  return PYIB_OK;
}

// Implicit direct forcing (ib_immersed.py:122-174): f solves (D S + eps I) f = rhs,
// D = interpolation (w hh^3), S = spreading (w ds^3), eps = 1e-8 tr(D S)/M.  With
// sq = sqrt(ds^3) the system is the symmetric positive definite
//   sq * D S (y / sq) + eps y = sq * rhs,   f = y / sq,
// solved by CG: the operator applies the device spreading and interpolation, the
// 3M-long marker vectors (the three components as one block-diagonal system) stay
// on the host, where the dot products are plain sequential sums.  rhs and the
// result are in ctx->dL; ctx->lag and ctx->conv are scratch.
int ib_implicit_solve(pyib_ctx* ctx) {
  const int M = ctx->M;
  const long long n = 3LL * M, nc = ctx->lay.ncell, tot = (long long)M * 125;
  std::vector<double> ds3(M), b(n), y(n, 0.0), r(n), p(n), ap(n), tmp(n);
  CK(cudaMemcpyAsync(ds3.data(), ctx->ds, M * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(b.data(), ctx->dL, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  double* dtr = ctx->partials + (size_t)(kSlots - 2) * kPartStride;   // one double of scratch
  k_ib_trace<<<grid_for(tot), kThreads, 0, ctx->stream>>>(tot, ctx->ibw, ctx->ds, ctx->partials, ctx->st, dtr);
  CKL();
  double trace = 0.0;
  CK(cudaMemcpyAsync(&trace, dtr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double eps = 1e-8 * (trace * ctx->prm.hh3) / M;
  std::vector<double> sq(M);
  for (int i = 0; i < M; ++i) sq[i] = std::sqrt(ds3[i]);
  auto apply = [&](const std::vector<double>& in, std::vector<double>& out) -> int {
    for (long long q = 0; q < n; ++q) tmp[q] = in[q] / sq[q / 3];
    CK(cudaMemcpyAsync(ctx->lag, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    RET(ib_spread(ctx, ctx->lag, ctx->conv));
    k_ib_interp<<<grid_for(M), kThreads, 0, ctx->stream>>>(M, nc, ctx->ibcell, ctx->ibw, ctx->prm.hh3, ctx->conv,
                                                          ctx->dL);
    CKL();
    CK(cudaMemcpyAsync(out.data(), ctx->dL, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (long long q = 0; q < n; ++q) out[q] = sq[q / 3] * out[q] + eps * in[q];
    return PYIB_OK;
  };
  double bb = 0.0;
  for (long long q = 0; q < n; ++q) {
    b[q] *= sq[q / 3];
    r[q] = b[q];
    p[q] = b[q];
    bb += b[q] * b[q];
  }
  double rr = bb;
  const double target = 1e-26 * bb;           // |r| <= 1e-13 |b|
  int it = 0;
  const int max_it = 2000;
  while (rr > target && it < max_it) {
    RET(apply(p, ap));
    double pap = 0.0;
    for (long long q = 0; q < n; ++q) pap += p[q] * ap[q];
    if (!(pap > 0.0)) return set_err(ctx, PYIB_E_NOCONV, "implicit IB solve: coupling matrix not positive");
    const double alpha = rr / pap;
    double rr_new = 0.0;
    for (long long q = 0; q < n; ++q) {
      y[q] += alpha * p[q];
      r[q] -= alpha * ap[q];
      rr_new += r[q] * r[q];
    }
    const double beta = rr_new / rr;
    for (long long q = 0; q < n; ++q) p[q] = r[q] + beta * p[q];
    rr = rr_new;
    ++it;
  }
  if (!(rr <= target))
    return set_err(ctx, PYIB_E_NOCONV, "implicit IB solve did not converge: %d iterations, |r|/|b| = %.3e", it,
                   std::sqrt(rr / (bb > 0.0 ? bb : 1.0)));
  for (long long q = 0; q < n; ++q) tmp[q] = y[q] / sq[q / 3];
  CK(cudaMemcpyAsync(ctx->dL, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  ctx->imp_iters = it;
  return PYIB_OK;
}

int ib_alloc(pyib_ctx* ctx, int M) {
  if (ctx->M == M && ctx->mk) return PYIB_OK;
  void* ptrs[] = {ctx->mk, ctx->mvel, ctx->ds, ctx->fL, ctx->lag, ctx->dL, ctx->ibw, ctx->ibcell,
                  ctx->ibbase, ctx->sort_keys_in, ctx->sort_keys_out, ctx->sort_vals_in,
                  ctx->sort_vals_out, ctx->sort_tmp, ctx->ibjac};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  ctx->M = M;
  const long long tot = (long long)M * 125;
  RET(alloc(ctx, (void**)&ctx->mk, 3 * M * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->mvel, 3 * M * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->ds, M * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->fL, 3 * M * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->lag, 3 * M * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->dL, 3 * M * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->ibw, tot * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->ibcell, tot * sizeof(int)));
  RET(alloc(ctx, (void**)&ctx->ibbase, 3 * M * sizeof(int)));
  RET(alloc(ctx, (void**)&ctx->ibjac, 9 * (long long)M * sizeof(double)));
  RET(alloc(ctx, (void**)&ctx->sort_keys_in, tot * sizeof(int)));
  RET(alloc(ctx, (void**)&ctx->sort_keys_out, tot * sizeof(int)));
  RET(alloc(ctx, (void**)&ctx->sort_vals_in, tot * sizeof(int)));
  RET(alloc(ctx, (void**)&ctx->sort_vals_out, tot * sizeof(int)));
  size_t tb = 0;
  CK(cub::DeviceRadixSort::SortPairs((void*)nullptr, tb, ctx->sort_keys_in, ctx->sort_keys_out,
                                     ctx->sort_vals_in, ctx->sort_vals_out, (int)tot, 0, 31,
                                     ctx->stream));
  ctx->sort_tmp_bytes = tb;
  RET(alloc(ctx, &ctx->sort_tmp, tb));
  ctx->stencil_valid = false;
  return PYIB_OK;
}

// ---- one step ------------------------------------------------------------
// One time step (Driver.step, ib_driver_np.py:412-532) in parts, so that a batch can
// run the Helmholtz solves of many cases together: step_begin (markers, held force,
// calc_vel, the explicit convection/diffusion part, the guess), then for each inner
// iteration step_rhs (force update of the direct mode, the residual, res_e), the
// solve, and step_after_solve (statistics, calc_vel, the accumulated force update).
struct StepRun {
  double dt = 0.0, dt_old = 0.0;
  int inner = 0, it = 0;
  bool accumulated = false, ib = false;
  pyib_step_stats st{};
};

int step_begin(pyib_ctx* ctx, StepRun& sr, double dt, double dt_old, int inner, const double* markers,
               const double* vel) {
  if (!tables_ready(ctx) || !ctx->have_params) return set_err(ctx, PYIB_E_STATE, "context not ready");
  sr = StepRun{};
  sr.dt = dt;
  sr.dt_old = dt_old;
  sr.inner = inner;
  sr.it = 1;
  sr.accumulated = ctx->prm.ib_mode == 0;
  if (sr.accumulated && inner < 2)
    return set_err(ctx, PYIB_E_ARG, "accumulated_explicit requires at least 2 fluid inner iterations");
  if (inner < 1) return set_err(ctx, PYIB_E_ARG, "at least one fluid inner iteration");
  const pyib_params& P = ctx->prm;
  const long long ne = ctx->lay.nedge;
  sr.ib = ctx->M > 0;
  sr.st.all_converged = 1;
  if (sr.ib && markers) {
    CK(cudaMemcpyAsync(ctx->mk, markers, 3 * ctx->M * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->mvel, vel, 3 * ctx->M * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    RET(ib_stencil(ctx));
    if (sr.accumulated) RET(ib_spread(ctx, ctx->fL, ctx->fE));   // held force follows the body (ib_driver_np.py:447-451)
  } else if (sr.ib && !ctx->stencil_valid) {
    RET(ib_stencil(ctx));
  }
  RET(op_calc_vel(ctx));
  const double rou = P.rou, ac = P.ac, ad = P.ad;
  RET(op_convdiff(ctx, 1, ((1.0 - ac) * dt) * rou, (1.0 - ad) * dt, dt, nullptr, nullptr, ctx->res_c0, nullptr));
  k_guess<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->s, ctx->s_old, ctx->prev, dt, dt_old);
  CKL();
  RET(op_calc_vel(ctx));
  return PYIB_OK;
}

int step_rhs(pyib_ctx* ctx, StepRun& sr) {
  const pyib_params& P = ctx->prm;
  const long long nc = ctx->lay.ncell;
  const double dt = sr.dt, rou = P.rou, ac = P.ac, ad = P.ad;
  if (sr.ib && !sr.accumulated) {
    // direct mode: this iteration's force replaces the last (ib_driver_np.py:466-486)
    RET(ib_interp(ctx, ctx->lag));
    k_ib_force<<<grid_for(3 * ctx->M), kThreads, 0, ctx->stream>>>(ctx->M, ctx->mvel, ctx->lag, dt, ctx->dL);
    CKL();
    if (ctx->prm.ib_mode == 2) RET(ib_implicit_solve(ctx));
    RET(ib_spread(ctx, ctx->dL, ctx->conv));   // conv is free scratch before op_convdiff
    const double ra = rou * ctx->prm.ib_alpha;
    k_set_scaled<<<grid_for(3 * nc), kThreads, 0, ctx->stream>>>(3 * nc, ctx->fE, ra, ctx->conv);
    CKL();
    k_set_scaled<<<grid_for(3 * ctx->M), kThreads, 0, ctx->stream>>>(3 * ctx->M, ctx->fL, ra, ctx->dL);
    CKL();
    sr.st.ib_updates += 1;
  }
  RET(op_convdiff(ctx, 2, (ac * dt) * rou, ad * dt, dt, ctx->res_c0, sr.ib ? ctx->fE : nullptr, ctx->res_c,
                  nullptr));
  RET(op_integr(ctx, ctx->res_c, nc, ctx->F));
  RET(op_rot(ctx, ctx->F, ctx->res_e));
  return PYIB_OK;
}

// statistics of this iteration's solve (kept when the solve failed), then the rest of
// the inner iteration; sr.it moves to the next one
int step_after_solve(pyib_ctx* ctx, StepRun& sr, const pyib_solve_stats& ss, int solve_rc, pyib_step_stats* out) {
  const long long nc = ctx->lay.ncell;
  const double rou = ctx->prm.rou;
  sr.st.max_iterations = ss.iterations > sr.st.max_iterations ? ss.iterations : sr.st.max_iterations;
  sr.st.total_iterations += ss.iterations;
  sr.st.max_rel_residual = fmax(sr.st.max_rel_residual, ss.rel_residual);
  sr.st.max_tol_ratio = fmax(sr.st.max_tol_ratio, ss.tol_ratio);
  sr.st.all_converged = sr.st.all_converged && ss.converged;
  if (out) *out = sr.st;
  if (solve_rc != PYIB_OK) return solve_rc;
  RET(op_calc_vel(ctx));
  if (sr.ib && sr.accumulated && sr.it == 1) {
    RET(ib_interp(ctx, ctx->lag));
    k_ib_force<<<grid_for(3 * ctx->M), kThreads, 0, ctx->stream>>>(ctx->M, ctx->mvel, ctx->lag, sr.dt, ctx->dL);
    CKL();
    RET(ib_spread(ctx, ctx->dL, ctx->conv));   // conv is free scratch here
    k_axpy_scaled<<<grid_for(3 * nc), kThreads, 0, ctx->stream>>>(3 * nc, ctx->fE, rou, ctx->conv);
    CKL();
    k_axpy_scaled<<<grid_for(3 * ctx->M), kThreads, 0, ctx->stream>>>(3 * ctx->M, ctx->fL, rou, ctx->dL);
    CKL();
    sr.st.ib_updates += 1;
  }
  ++sr.it;
  return PYIB_OK;
}

int step_end(pyib_ctx* ctx, StepRun& sr, pyib_step_stats* out) {
  RET(check_dev_err(ctx));
  if (out) *out = sr.st;
  return PYIB_OK;
}

int do_step(pyib_ctx* ctx, double dt, double dt_old, int inner, const double* markers, const double* vel,
            pyib_step_stats* out) {
  StepRun sr;
  RET(step_begin(ctx, sr, dt, dt_old, inner, markers, vel));
  while (sr.it <= sr.inner) {
    RET(step_rhs(ctx, sr));
    pyib_solve_stats ss{};
    const int rc = ctx->prm.precision == 1 ? helm_solve_mixed(ctx, dt, &ss) : helm_solve(ctx, dt, &ss);
    RET(step_after_solve(ctx, sr, ss, rc, out));
  }
  return step_end(ctx, sr, out);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
// Times reps back-to-back matvecs in -> out, then each of its kernels alone (benchmark
// support for pyib_bench_matvec).
template <typename T>
int bench_matvec_t(pyib_ctx* ctx, int reps, const T* in, T* out, T* vcm, T* vq, const T* pa, const T* pv,
                   const T* pr, double* ms_per) {
  RET(launch_matvec_t<T>(ctx, in, out, vcm, vq, in, 1, 0, pa, pv, pr));   // warm
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  for (int q = 0; q < reps; ++q) RET(launch_matvec_t<T>(ctx, in, out, vcm, vq, in, 1, 0, pa, pv, pr));
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ms_per[0] = ms / reps;
  // each kernel alone, same inputs (after a full matvec, so every intermediate is current)
  const Meta& m = sizeof(T) == 4 ? ctx->meta32 : ctx->meta;
  const long long nc = ctx->lay.ncell;
  const dim3 blk(TX, TY, 1), gA(m.gxA, m.gyA, m.gzA), gV(m.gxV, m.gyA, m.gzA), gR(m.gxR, m.gyR, m.gzR);
  for (int kern = 0; kern < 6; ++kern) {
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int q = 0; q < reps; ++q) {
      switch (kern) {
        case 0:
          if (m.av)
            k_mvAV<T><<<gA, blk, 0, ctx->stream>>>(m, in, vcm, vq, ctx->f_flags, ctx->st);
          else
            k_mvA<T><<<gA, blk, 0, ctx->stream>>>(m, in, vcm, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                  ctx->nA, ctx->st);
          break;
        case 1: k_patchA<T><<<patch_grid(3 * ctx->nA), kThreads, 0, ctx->stream>>>(
                    ctx->nA, tp<int>(ctx, PYIB_T_PA_IDS), tp<long long>(ctx, PYIB_T_PA_PTR),
                    tp<int>(ctx, PYIB_T_PA_COL), pa, in, vcm, nc, ctx->st); break;
        case 2:
          if (m.av) continue;   // fused into kernel AV (slot 1)
          k_mvV<T><<<gV, blk, 0, ctx->stream>>>(m, vcm, vq, ctx->st);
          break;
        case 3: k_patchV<T><<<patch_grid(ctx->nV), kThreads, 0, ctx->stream>>>(
                    ctx->nV, tp<int>(ctx, PYIB_T_PV_IDS), tp<long long>(ctx, PYIB_T_PV_PTR),
                    tp<int>(ctx, PYIB_T_PV_COL), pv, vcm, vq, nc, ctx->st); break;
        case 4: k_mvRI<T><<<gR, blk, 0, ctx->stream>>>(m, vq, out, in, tp<unsigned int>(ctx, PYIB_T_PR_BITS),
                                                       ctx->partials, ctx->st, 1); break;
        default: k_patchRI<T><<<patch_grid(ctx->nR), kThreads, 0, ctx->stream>>>(
                    ctx->nR, tp<int>(ctx, PYIB_T_PR_IDS), tp<long long>(ctx, PYIB_T_PR_PTR),
                    tp<int>(ctx, PYIB_T_PR_COL), pr, vq, out, in, ctx->partials, m.nplanes, ctx->st, 1); break;
      }
      CKL();
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ms_per[1 + kern] = ms / reps;
  }
  return PYIB_OK;
}

// Carves 256-byte aligned pieces out of one buffer; with base == nullptr it only
// adds up the size.
struct Carve {
  char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
};

// grows *buf to at least bytes (the stream is drained first: the old buffer may be in use)
static int grow(pyib_ctx* ctx, void** buf, size_t* have, size_t bytes) {
  if (bytes <= *have && *buf) return PYIB_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *have = 0;
  CK(cudaMalloc(buf, bytes < 256 ? 256 : bytes));
  *have = bytes < 256 ? 256 : bytes;
  return PYIB_OK;
}

// Jacobi PCG from zero on a device CSR (three kernels per iteration).  Chunks of
// 16 iterations between reads of the state; kernels after convergence return at once.
static int graph_cg(pyib_ctx* ctx, long long n, const long long* ptr, const int* col, const double* val,
                    const double* b, const double* dinv, double* x, double* r, double* z, double* p, double* q,
                    double rtol, int max_iterations, double* parts, GState* gs, GState& h) {
  cudaStream_t st = ctx->stream;
  CK(cudaEventRecord(ctx->ev0, st));
  k_g_init<<<grid_for(n), kThreads, 0, st>>>(n, rtol, b, dinv, x, r, z, p, parts, gs);
  CKL();
  CK(cudaMemcpyAsync(&h, gs, sizeof(GState), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  int launched = 0;
  while (!h.done && launched < max_iterations) {
    const int chunk = std::min(16, max_iterations - launched);
    for (int c = 0; c < chunk; ++c) {
      k_g_mvpq<<<grid_for(n), kThreads, 0, st>>>(n, ptr, col, val, p, q, parts, gs);
      CKL();
      // 40 registers: 6 resident blocks per SM, so one wave of 148 x 6 blocks
      k_g_update<<<std::min(grid_for(n), 148 * 6), kThreads, 0, st>>>(n, p, q, dinv, x, r, z, parts, gs);
      CKL();
      k_g_p<<<grid_for(n), kThreads, 0, st>>>(n, z, p, gs);
      CKL();
    }
    launched += chunk;
    CK(cudaMemcpyAsync(&h, gs, sizeof(GState), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (!std::isfinite(h.rr)) return set_err(ctx, PYIB_E_NONFINITE, "graph PCG: non-finite residual");
  }
  CK(cudaEventRecord(ctx->ev1, st));
  return PYIB_OK;
}

// ---------------------------------------------------------------------------
// Batches: independent cases on one GPU whose CG iterations run together, one launch
// per kernel stage over the tiles of every case still iterating (k_b* kernels),
// `check` iterations to a CUDA graph.  Everything else of a step runs per case on the
// case's own stream, through the same step parts as pyib_step.
// ---------------------------------------------------------------------------
struct pyib_batch {
  std::vector<pyib_ctx*> cs;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  BCase* d_cases = nullptr;        // one per case, in the precision of the current solve
  int2* d_blk = nullptr;           // (case, block within the case's grid) of every block of every stage
  size_t blk_cap = 0;              // int2 entries d_blk holds
  std::vector<BCase> h_cases;
  std::vector<int2> h_blk;
  // stage q of group g: h_blk[blk_off[g][q] .. blk_off[g][q+1])
  long long blk_off[kBatchGroups][kBStages + 1] = {};
  cudaStream_t gstream[kBatchGroups] = {};     // capture branches of the groups
  cudaEvent_t fork = nullptr, join[kBatchGroups] = {};
  cudaGraphExec_t graph = nullptr;
  std::vector<char> graph_for;     // the iterating cases the graph was captured for
  int graph_prec = -1;
  long long graph_kernels = 0;     // kernel nodes of one replay
  long long launches = 0;          // batched kernels launched (replays x kernel nodes)
  long long captures = 0;          // graph captures
  double chunk_seconds = 0.0;      // CUDA-event time of the batched chunks
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

static int batch_err(pyib_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  b->err = buf;
  return code;
}

#define BCK(call)                                                                      \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return batch_err(b, PYIB_E_CUDA, "%s failed: %s (%s:%d)", #call,                 \
                       cudaGetErrorString(e_), __FILE__, __LINE__);                    \
  } while (0)

// a failing case's status, with its message as the batch's
static int batch_case_rc(pyib_batch* b, int c, int rc) {
  if (rc != PYIB_OK) b->err = "case " + std::to_string(c) + ": " + b->cs[c]->err;
  return rc;
}

// the device view of case c for a solve in float64 (prec 0) or float32 (prec 1)
static BCase batch_view(pyib_ctx* ctx, int prec) {
  BCase q{};
  q.m = prec ? ctx->meta32 : ctx->meta;
  q.st = ctx->st;
  q.partials = ctx->partials;
  if (prec) {
    q.p = ctx->p32; q.w = ctx->w32; q.vcm = ctx->vcm32; q.vq = ctx->vq32; q.r = ctx->r32; q.x = ctx->x32;
    q.pa_val = ctx->pa_val32; q.pv_val = ctx->pv_val32; q.pr_val = ctx->pr_val32;
  } else {
    q.p = ctx->p; q.w = ctx->w; q.vcm = ctx->vcm; q.vq = ctx->vq; q.r = ctx->r; q.x = ctx->x;
    q.pa_val = tp<double>(ctx, PYIB_T_PA_VAL); q.pv_val = tp<double>(ctx, PYIB_T_PV_VAL);
    q.pr_val = tp<double>(ctx, PYIB_T_PR_VAL);
  }
  q.pa_ids = tp<int>(ctx, PYIB_T_PA_IDS); q.pa_col = tp<int>(ctx, PYIB_T_PA_COL);
  q.pv_ids = tp<int>(ctx, PYIB_T_PV_IDS); q.pv_col = tp<int>(ctx, PYIB_T_PV_COL);
  q.pr_ids = tp<int>(ctx, PYIB_T_PR_IDS); q.pr_col = tp<int>(ctx, PYIB_T_PR_COL);
  q.pa_ptr = tp<long long>(ctx, PYIB_T_PA_PTR); q.pv_ptr = tp<long long>(ctx, PYIB_T_PV_PTR);
  q.pr_ptr = tp<long long>(ctx, PYIB_T_PR_PTR);
  q.prec_bits = tp<unsigned int>(ctx, PYIB_T_PREC_BITS);
  q.pr_bits = tp<unsigned int>(ctx, PYIB_T_PR_BITS);
  q.prec = tp<double>(ctx, PYIB_T_PREC);
  q.dinv = ctx->prec32;
  q.nA = ctx->nA; q.nV = ctx->nV; q.nR = ctx->nR;
  q.ne = ctx->lay.nedge; q.nc = ctx->lay.ncell;
  // Deep z-chunks for the batched tiles: a batched block first looks up its case, so
  // longer blocks amortise that.  The cell kernels compute cell by cell and the dot's
  // partials are indexed by plane, so the depths change no result.
  set_grids(q.m, kBatchCellDepth, kBatchNodeDepth);
  const Meta& m = q.m;
  q.nblk[0] = m.gxA * m.gyA * m.gzA;
  q.nblk[1] = q.nA > 0 ? patch_grid(3 * q.nA) : 0;
  q.nblk[2] = m.gxV * m.gyA * m.gzA;
  q.nblk[3] = q.nV > 0 ? patch_grid(q.nV) : 0;
  q.nblk[4] = m.gxR * m.gyR * m.gzR;
  q.nblk[5] = patch_grid(q.nR);        // also the final reduction of p.w
  q.nblk[6] = grid_for(q.ne);
  q.nblk[7] = grid_for(q.ne);
  return q;
}

// The iterating cases in kBatchGroups groups of about equal work (edges; largest
// first, each to the lightest group), and the block table of every stage of every
// group: the blocks of each case's own grids, so every reduction sums in the case's
// own order.
static int batch_blocks(pyib_batch* b, const std::vector<char>& on) {
  const int n = (int)b->cs.size();
  std::vector<int> order;
  for (int c = 0; c < n; ++c)
    if (on[c]) order.push_back(c);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return b->h_cases[x].ne > b->h_cases[y].ne; });
  std::vector<int> group(n, -1);
  long long load[kBatchGroups] = {0};
  for (int c : order) {
    int g = 0;
    for (int k = 1; k < kBatchGroups; ++k)
      if (load[k] < load[g]) g = k;
    group[c] = g;
    load[g] += b->h_cases[c].ne;
  }
  b->h_blk.clear();
  for (int g = 0; g < kBatchGroups; ++g) {
    for (int q = 0; q < kBStages; ++q) {
      b->blk_off[g][q] = (long long)b->h_blk.size();
      for (int c = 0; c < n; ++c)
        if (group[c] == g)
          for (int k = 0; k < b->h_cases[c].nblk[q]; ++k) b->h_blk.push_back(make_int2(c, k));
    }
    b->blk_off[g][kBStages] = (long long)b->h_blk.size();
  }
  if (b->h_blk.size() > b->blk_cap) {
    if (b->d_blk) BCK(cudaFree(b->d_blk));
    b->d_blk = nullptr;
    b->blk_cap = 0;
    BCK(cudaMalloc((void**)&b->d_blk, b->h_blk.size() * sizeof(int2)));
    b->blk_cap = b->h_blk.size();
  }
  if (!b->h_blk.empty())
    BCK(cudaMemcpyAsync(b->d_blk, b->h_blk.data(), b->h_blk.size() * sizeof(int2), cudaMemcpyHostToDevice,
                        b->stream));
  return PYIB_OK;
}

// (Re)captures the chunk graph: `check` iterations of the 8 stages over the cases in on.
static int batch_graph(pyib_batch* b, int prec, const std::vector<char>& on) {
  if (b->graph && b->graph_prec == prec && b->graph_for == on) return PYIB_OK;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  RET(batch_blocks(b, on));
  BCK(cudaStreamSynchronize(b->stream));   // the block table is in place before any branch reads it
  const int check = b->cs[0]->prm.check;
  cudaGraph_t g;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  const dim3 blk2(TX, TY, 1);
  // errors inside the capture are kept until it has ended, so the stream never stays capturing
  cudaError_t ce = cudaEventRecord(b->fork, b->stream);
  for (int grp = 0; grp < kBatchGroups; ++grp) {
   if (b->blk_off[grp][kBStages] == b->blk_off[grp][0]) continue;
   cudaStream_t gs = b->gstream[grp];
   if (ce == cudaSuccess) ce = cudaStreamWaitEvent(gs, b->fork, 0);
   for (int it = 0; it < check; ++it) {
    for (int q = 0; q < kBStages; ++q) {
      const int total = (int)(b->blk_off[grp][q + 1] - b->blk_off[grp][q]);
      if (total == 0) continue;
      const int2* st = b->d_blk + b->blk_off[grp][q];
      if (prec) {
        switch (q) {
          case 0: k_bA<float><<<total, blk2, 0, gs>>>(b->d_cases, st); break;
          case 1: k_bpatchA<float><<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
          case 2: k_bV<float><<<total, blk2, 0, gs>>>(b->d_cases, st); break;
          case 3: k_bpatchV<float><<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
          case 4: k_bRI<float><<<total, blk2, 0, gs>>>(b->d_cases, st); break;
          case 5: k_bpatchRI<float><<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
          case 6: k_bupdate32<<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
          default: k_bdir32<<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
        }
      } else {
        switch (q) {
          case 0: k_bA<double><<<total, blk2, 0, gs>>>(b->d_cases, st); break;
          case 1: k_bpatchA<double><<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
          case 2: k_bV<double><<<total, blk2, 0, gs>>>(b->d_cases, st); break;
          case 3: k_bpatchV<double><<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
          case 4: k_bRI<double><<<total, blk2, 0, gs>>>(b->d_cases, st); break;
          case 5: k_bpatchRI<double><<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
          case 6: k_bupdate<<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
          default: k_bdir<<<total, kThreads, 0, gs>>>(b->d_cases, st); break;
        }
      }
    }
   }
   if (ce == cudaSuccess) ce = cudaEventRecord(b->join[grp], gs);
   if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->stream, b->join[grp], 0);
  }
  const cudaError_t le = cudaGetLastError();
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (ce != cudaSuccess || e != cudaSuccess) {
    if (e == cudaSuccess) cudaGraphDestroy(g);
    return batch_err(b, PYIB_E_CUDA, "batch graph capture failed: %s",
                     cudaGetErrorString(ce != cudaSuccess ? ce : e));
  }
  if (le != cudaSuccess) {
    cudaGraphDestroy(g);
    return batch_err(b, PYIB_E_CUDA, "batched launch failed: %s", cudaGetErrorString(le));
  }
  b->graph_kernels = graph_kernels(g);
  const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return batch_err(b, PYIB_E_CUDA, "batch graph instantiate failed: %s", cudaGetErrorString(ie));
  b->graph_prec = prec;
  b->graph_for = on;
  ++b->captures;
  return PYIB_OK;
}

// Replays the chunk graph over the cases in on, then reads every iterating case's
// state (one copy each, one synchronisation).
static int batch_chunk(pyib_batch* b, int prec, const std::vector<char>& on) {
  RET(batch_graph(b, prec, on));
  BCK(cudaEventRecord(b->ev0, b->stream));
  BCK(cudaGraphLaunch(b->graph, b->stream));
  BCK(cudaEventRecord(b->ev1, b->stream));
  b->launches += b->graph_kernels;
  for (size_t c = 0; c < b->cs.size(); ++c)
    if (on[c])
      BCK(cudaMemcpyAsync(b->cs[c]->st_host, b->cs[c]->st, sizeof(CGState), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  float ms = 0.f;
  BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->chunk_seconds += ms * 1e-3;
  return PYIB_OK;
}

// One Helmholtz solve of every case (helm_solve or helm_solve_mixed), the CG
// iterations of all cases batched.  rc[c] is case c's status; the batch's own
// failures (CUDA errors of the batched launches) are returned.
static int batch_solve(pyib_batch* b, const std::vector<double>& dt, std::vector<pyib_solve_stats>& ss,
                       std::vector<int>& rc) {
  const int n = (int)b->cs.size();
  const int prec = b->cs[0]->prm.precision == 1 ? 1 : 0;
  std::vector<char> on(n, 0);
  std::vector<MixRun> mr(n);
  std::vector<long long> chunks(n, 0);
  std::vector<char> iterated(n, 0);
  for (int c = 0; c < n; ++c) {
    pyib_ctx* ctx = b->cs[c];
    if (rc[c] != PYIB_OK) continue;
    bool it = false;
    rc[c] = prec ? mixed_begin(ctx, dt[c], false, mr[c], &it) : solve_begin(ctx, dt[c], false, &it);
    if (rc[c] == PYIB_OK) BCK(cudaStreamSynchronize(ctx->stream));   // its start is in place before the chunks
    on[c] = rc[c] == PYIB_OK && it;
    iterated[c] = on[c];
    b->h_cases[c] = batch_view(ctx, prec);
  }
  BCK(cudaMemcpyAsync(b->d_cases, b->h_cases.data(), n * sizeof(BCase), cudaMemcpyHostToDevice, b->stream));
  for (;;) {
    bool any = false;
    for (int c = 0; c < n; ++c) any = any || on[c];
    if (!any) break;
    RET(batch_chunk(b, prec, on));
    for (int c = 0; c < n; ++c) {
      if (!on[c]) continue;
      pyib_ctx* ctx = b->cs[c];
      ++chunks[c];
      if (!ctx->st_host->done && chunks[c] < max_cg_chunks(ctx)) continue;
      if (prec) {
        // the float32 CG stopped: fold its correction into x and decide
        bool more = false;
        rc[c] = mixed_refine(ctx, mr[c], &more);
        if (rc[c] == PYIB_OK) BCK(cudaStreamSynchronize(ctx->stream));
        on[c] = rc[c] == PYIB_OK && more;
        chunks[c] = 0;
      } else {
        on[c] = 0;
      }
    }
  }
  for (int c = 0; c < n; ++c) {
    if (rc[c] != PYIB_OK) continue;
    pyib_ctx* ctx = b->cs[c];
    rc[c] = prec ? mixed_end(ctx, mr[c], &ss[c]) : solve_end(ctx, iterated[c] != 0, &ss[c]);
  }
  return PYIB_OK;
}

// One time step of every case (do_step), the Helmholtz solves batched.
static int batch_step(pyib_batch* b, const double* dt, const double* dt_old, int inner,
                      const double* const* markers, const double* const* vel, pyib_step_stats* stats) {
  const int n = (int)b->cs.size();
  std::vector<StepRun> sr(n);
  std::vector<int> rc(n, PYIB_OK);
  std::vector<double> dts(dt, dt + n);
  for (int c = 0; c < n; ++c) {
    pyib_ctx* ctx = b->cs[c];
    RET(batch_case_rc(b, c, step_begin(ctx, sr[c], dt[c], dt_old[c], inner, markers ? markers[c] : nullptr,
                                       vel ? vel[c] : nullptr)));
  }
  for (int it = 1; it <= inner; ++it) {
    for (int c = 0; c < n; ++c) RET(batch_case_rc(b, c, step_rhs(b->cs[c], sr[c])));
    std::vector<pyib_solve_stats> ss(n);
    RET(batch_solve(b, dts, ss, rc));
    for (int c = 0; c < n; ++c)
      RET(batch_case_rc(b, c, step_after_solve(b->cs[c], sr[c], ss[c], rc[c], stats ? &stats[c] : nullptr)));
  }
  for (int c = 0; c < n; ++c) RET(batch_case_rc(b, c, step_end(b->cs[c], sr[c], stats ? &stats[c] : nullptr)));
  return PYIB_OK;
}

extern "C" {

int pyib_version(char* buf, size_t n) {
  if (!buf || n == 0) return PYIB_E_ARG;
  snprintf(buf, n, "%s", PYIB_VERSION);
  return PYIB_OK;
}

int pyib_last_error(const pyib_ctx* ctx, char* buf, size_t n) {
  if (!ctx || !buf || n == 0) return PYIB_E_ARG;
  snprintf(buf, n, "%s", ctx->err.c_str());
  return PYIB_OK;
}

int pyib_create(const pyib_layout* layout, pyib_ctx** out) {
  if (!layout || !out) return PYIB_E_ARG;
  *out = nullptr;
  if (layout->nlevels < 1 || layout->nlevels > PYIB_MAX_LEVELS) return PYIB_E_ARG;
  pyib_ctx* ctx = new pyib_ctx();
  ctx->lay = *layout;
  ctx->device = layout->device;
  // meta
  Meta& m = ctx->meta;
  m.nl = layout->nlevels;
  m.ri_up = 1;                     // until pyib_finalize knows the upper faces are exact
  long long cb = 0, fb = 0, eb = 0;
  for (int L = 0; L < m.nl; ++L) {
    LevelMeta& l = m.lv[L];
    for (int a = 0; a < 3; ++a) {
      l.n[a] = layout->n[L][a];
      l.hole_lo[a] = layout->hole_lo[L][a];
      l.hole_hi[a] = layout->hole_lo[L][a] + layout->hole_n[L][a];
    }
    l.has_hole = layout->hole_n[L][0] > 0;
    l.h = layout->h[L];
    l.cbase = cb;
    cb += (long long)l.n[0] * l.n[1] * l.n[2];
  }
  for (int L = 0; L < m.nl; ++L) {
    LevelMeta& l = m.lv[L];
    for (int a = 0; a < 3; ++a) {
      l.fbase[a] = fb;
      fb += (long long)(l.n[0] + (a == 0)) * (l.n[1] + (a == 1)) * (l.n[2] + (a == 2));
    }
  }
  for (int L = 0; L < m.nl; ++L) {
    LevelMeta& l = m.lv[L];
    for (int a = 0; a < 3; ++a) {
      l.ebase[a] = eb;
      l.ecount[a] = (long long)(l.n[0] + (a != 0)) * (l.n[1] + (a != 1)) * (l.n[2] + (a != 2));
      eb += l.ecount[a];
    }
  }
  m.nc = cb; m.nf = fb; m.ne = eb;
  set_grids_fused(m, 16);
  {
    const char* f = std::getenv("PYIB_FUSED_MATVEC");
    ctx->use_fused = f && f[0] == '1';
    const char* av = std::getenv("PYIB_MATVEC_AV");
    ctx->av_pin = (av && av[0] == '0') ? 0 : (av && av[0] == '1') ? 1 : -1;
  }
  {
    // default z-chunk depth: the deepest of 16, 8, 4, 2, 1 planes that still yields
    // enough tiles (the autotuner may change it, see tune_matvec)
    long long plane_tiles = 0;
    for (int L = 0; L < m.nl; ++L) {
      const LevelMeta& l = m.lv[L];
      plane_tiles += (long long)((l.n[0] + TX - 1) / TX) * ((l.n[1] + TY - 1) / TY) * l.n[2];
    }
    int kz = 16;
    while (kz > 1 && plane_tiles / kz < kTargetBlocks) kz >>= 1;
    set_grids(m, kz, kz);
    if ((long long)m.gxR * m.gyR * m.gzR > kPartStride) {
      delete ctx;
      return PYIB_E_ARG;
    }
  }
  if (cb != layout->ncell || fb != layout->nface || eb != layout->nedge) {
    delete ctx;
    return PYIB_E_ARG;
  }
  if (eb >= (1LL << 31) || cb * 3 >= (1LL << 31)) {
    delete ctx;
    return PYIB_E_ARG;
  }
  int rc = [&]() -> int {
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ctx->ev0));
    CK(cudaEventCreate(&ctx->ev1));
    const long long nc = cb, nf = fb, ne = eb, ncx = cb + layout->nbface;
    double** e_fields[] = {&ctx->s, &ctx->s_old, &ctx->res_e, &ctx->work_e, &ctx->work_e2, &ctx->x,
                           &ctx->r, &ctx->p, &ctx->w, &ctx->prev};
    for (double** f : e_fields) RET(alloc(ctx, (void**)f, ne * sizeof(double)));
    double** f_fields[] = {&ctx->U, &ctx->F, &ctx->work_f};
    for (double** f : f_fields) RET(alloc(ctx, (void**)f, nf * sizeof(double)));
    RET(alloc(ctx, (void**)&ctx->vc, 3 * ncx * sizeof(double)));
    double** c3_fields[] = {&ctx->res_c0, &ctx->res_c, &ctx->fE, &ctx->conv, &ctx->diff, &ctx->work_c3,
                            &ctx->vcm, &ctx->vq};
    for (double** f : c3_fields) RET(alloc(ctx, (void**)f, 3 * nc * sizeof(double)));
    RET(alloc(ctx, (void**)&ctx->partials, (size_t)kSlots * kPartStride * sizeof(double)));
    RET(alloc(ctx, (void**)&ctx->st, sizeof(CGState)));
    CK(cudaMallocHost((void**)&ctx->st_host, sizeof(CGState)));
    RET(alloc(ctx, (void**)&ctx->dev_err, sizeof(int)));
    CK(cudaStreamSynchronize(ctx->stream));
    return PYIB_OK;
  }();
  if (rc != PYIB_OK) {
    // keep ctx so the caller can read the error, then destroy
    *out = ctx;
    return rc;
  }
  *out = ctx;
  return PYIB_OK;
}

int pyib_destroy(pyib_ctx* ctx) {
  if (!ctx) return PYIB_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->cg_graph) cudaGraphExecDestroy(ctx->cg_graph);
  if (ctx->mix_graph) cudaGraphExecDestroy(ctx->mix_graph);
  for (auto& t : ctx->tab)
    if (t.ptr) cudaFree(t.ptr);
  void* ptrs[] = {ctx->s, ctx->s_old, ctx->U, ctx->vc, ctx->res_c0, ctx->res_c, ctx->res_e, ctx->F,
                  ctx->fE, ctx->conv, ctx->diff, ctx->work_e, ctx->work_e2, ctx->work_c3, ctx->work_f,
                  ctx->x, ctx->r, ctx->p, ctx->w, ctx->vcm, ctx->vq, ctx->prev, ctx->partials, ctx->st,
                  ctx->dev_err, ctx->mk, ctx->mvel, ctx->ds, ctx->fL, ctx->lag, ctx->dL, ctx->ibw,
                  ctx->ibcell, ctx->ibbase, ctx->sort_keys_in, ctx->sort_keys_out, ctx->sort_vals_in,
                  ctx->sort_vals_out, ctx->sort_tmp, ctx->x32, ctx->r32, ctx->p32, ctx->w32,
                  ctx->vcm32, ctx->vq32, ctx->prec32, ctx->pa_val32, ctx->pv_val32,
                  ctx->pr_val32, ctx->diag1, ctx->diag2, ctx->ibjac, ctx->ws, ctx->ws_tmp,
                  ctx->f_irrA, ctx->f_irrV, ctx->f_needR, ctx->f_list, ctx->f_flags};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (ctx->st_host) cudaFreeHost(ctx->st_host);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->tev0) cudaEventDestroy(ctx->tev0);
  if (ctx->tev1) cudaEventDestroy(ctx->tev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return PYIB_OK;
}

int pyib_upload(pyib_ctx* ctx, int32_t table, const void* host, size_t bytes) {
  if (!ctx || table < 0 || table >= PYIB_T_COUNT || (bytes && !host)) return PYIB_E_ARG;
  if (bytes % table_elem(table)) return set_err(ctx, PYIB_E_ARG, "table %d: %zu bytes is not a multiple of %zu",
                                                table, bytes, table_elem(table));
  CK(cudaSetDevice(ctx->device));
  Table& t = ctx->tab[table];
  if (t.ptr) {
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaFree(t.ptr));
    t.ptr = nullptr;
  }
  RET(alloc(ctx, &t.ptr, bytes));
  t.bytes = bytes;
  if (bytes) CK(cudaMemcpyAsync(t.ptr, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (table == PYIB_T_PA_VAL || table == PYIB_T_PV_VAL || table == PYIB_T_PR_VAL) {
    float** f = table == PYIB_T_PA_VAL ? &ctx->pa_val32 : (table == PYIB_T_PV_VAL ? &ctx->pv_val32 : &ctx->pr_val32);
    if (*f) { cudaFree(*f); *f = nullptr; }
    if (ctx->r32) {
      const long long n = (long long)(bytes / 8);
      RET(alloc(ctx, (void**)f, (n > 0 ? n : 1) * sizeof(float)));
      if (n > 0) { k_d2f<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, (const double*)t.ptr, *f); CKL(); }
    }
  }
  if (table == PYIB_T_PREC_REG) {
    if (bytes != (size_t)ctx->meta.nl * 8) return set_err(ctx, PYIB_E_ARG, "PREC_REG needs one value per level");
    for (int L = 0; L < ctx->meta.nl; ++L) ctx->meta.lv[L].prec_reg = ((const double*)host)[L];
  }
  if (table == PYIB_T_INLET_IDX) ctx->n_inlet = bytes / 4;
  if (table == PYIB_T_BF_FACE) ctx->n_bf = bytes / 4;
  if (table == PYIB_T_LC_CAND) ctx->n_cand = bytes / 4;
  if (table == PYIB_T_LC_FIDX) ctx->n_fidx = bytes / 4;
  ctx->cg_graph_check = -1;  // tables changed: recapture
  ctx->mix_graph_check = -1;
  ctx->diag_ready = false;
  ctx->diag_for_kfac = -1.0;
  ctx->tuned = false;
  ctx->tuned32 = false;
  ctx->tunedF = false;
  ctx->fused_ready = false;
  ctx->flags_ready = false;
  return PYIB_OK;
}

int pyib_finalize(pyib_ctx* ctx, const int64_t* counts, int32_t ncounts) {
  if (!ctx || !counts || ncounts < 3) return PYIB_E_ARG;
  ctx->nA = counts[0];
  ctx->nV = counts[1];
  ctx->nR = counts[2];
  ctx->meta.ri_up = (ncounts >= 4 && counts[3] != 0) ? 0 : 1;
  set_grids(ctx->meta, ctx->meta.kz, ctx->meta.kzR);
  set_grids_fused(ctx->meta, ctx->meta.kzF > 0 ? ctx->meta.kzF : 16);
  ctx->tuned32 = false;
  ctx->tunedF = false;
  ctx->fused_ready = false;
  ctx->flags_ready = false;
  if ((long long)ctx->meta.gxR * ctx->meta.gyR * ctx->meta.gzR + patch_grid(ctx->nR) > kPartStride ||
      (long long)ctx->meta.nplanes + patch_grid(ctx->nR) > kPartStride)
    return set_err(ctx, PYIB_E_ARG, "too many reduction slots for this layout");
  if (ctx->n_bf != ctx->lay.nbface)
    return set_err(ctx, PYIB_E_ARG, "boundary face table has %lld rows, layout says %d", ctx->n_bf,
                   ctx->lay.nbface);
  return PYIB_OK;
}

int pyib_set_params(pyib_ctx* ctx, const pyib_params* p) {
  if (!ctx || !p) return PYIB_E_ARG;
  if (p->check <= 0 || p->cg_max <= 0) return set_err(ctx, PYIB_E_ARG, "check and cg_max must be positive");
  if (p->nmarkers < 0) return set_err(ctx, PYIB_E_ARG, "negative marker count");
  CK(cudaSetDevice(ctx->device));
  const bool recapture = !ctx->have_params || ctx->prm.check != p->check;
  ctx->prm = *p;
  ctx->have_params = true;
  if (recapture) {
    ctx->cg_graph_check = -1;
    ctx->mix_graph_check = -1;
  }
  if (p->precision != 0 && p->precision != 1) return set_err(ctx, PYIB_E_ARG, "precision must be 0 or 1");
  if (p->ib_mode < 0 || p->ib_mode > 2) return set_err(ctx, PYIB_E_ARG, "ib_mode must be 0, 1 or 2");
  if (p->ib_mode != 0 && !(p->ib_alpha > 0.0)) return set_err(ctx, PYIB_E_ARG, "ib_alpha must be positive");
  if (p->nmarkers > 0) RET(ib_alloc(ctx, p->nmarkers));
  return PYIB_OK;
}

int pyib_set_ib_geometry(pyib_ctx* ctx, const double* pos_ref, double dx) {
  if (!ctx || !pos_ref || !(dx > 0)) return PYIB_E_ARG;
  for (int a = 0; a < 3; ++a) ctx->pos_ref[a] = pos_ref[a];
  ctx->dx = dx;
  for (int a = 0; a < 3; ++a) ctx->ib_n[a] = ctx->lay.n[0][a];
  ctx->stencil_valid = false;
  return PYIB_OK;
}

static int field_ptr(pyib_ctx* ctx, int32_t f, void** ptr, size_t* count, size_t* elem, bool* writable) {
  const long long nc = ctx->lay.ncell, ne = ctx->lay.nedge, nf = ctx->lay.nface, M = ctx->M;
  const long long ncx = ncx_of(ctx);
  *elem = 8;
  *writable = true;
  switch (f) {
    case PYIB_F_S: *ptr = ctx->s; *count = ne; break;
    case PYIB_F_S_OLD: *ptr = ctx->s_old; *count = ne; break;
    case PYIB_F_U: *ptr = ctx->U; *count = nf; break;
    case PYIB_F_VC: *ptr = ctx->vc; *count = 3 * ncx; break;   // component stride ncell+nbface
    case PYIB_F_VC_GHOST: *ptr = ctx->vc; *count = 3 * ncx; break;
    case PYIB_F_RES_C: *ptr = ctx->res_c; *count = 3 * nc; break;
    case PYIB_F_RES_E: *ptr = ctx->res_e; *count = ne; break;
    case PYIB_F_FE: *ptr = ctx->fE; *count = 3 * nc; break;
    case PYIB_F_FL: *ptr = ctx->fL; *count = 3 * M; break;
    case PYIB_F_MARKERS: *ptr = ctx->mk; *count = 3 * M; break;
    case PYIB_F_MVEL: *ptr = ctx->mvel; *count = 3 * M; break;
    case PYIB_F_DS: *ptr = ctx->ds; *count = M; break;
    case PYIB_F_WORK_E: *ptr = ctx->work_e; *count = ne; break;
    case PYIB_F_WORK_E2: *ptr = ctx->work_e2; *count = ne; break;
    case PYIB_F_WORK_C3: *ptr = ctx->work_c3; *count = 3 * nc; break;
    case PYIB_F_WORK_F: *ptr = ctx->work_f; *count = nf; break;
    case PYIB_F_IB_CELL: *ptr = ctx->ibcell; *count = 125 * M; *elem = 4; *writable = false; break;
    case PYIB_F_IB_W: *ptr = ctx->ibw; *count = 125 * M; *writable = false; break;
    case PYIB_F_IB_BASE: *ptr = ctx->ibbase; *count = 3 * M; *elem = 4; *writable = false; break;
    case PYIB_F_LAG_TMP: *ptr = ctx->lag; *count = 3 * M; break;
    case PYIB_F_DINV: *ptr = ctx->prec32; *count = ne; *elem = 4; *writable = false; break;
    default: return set_err(ctx, PYIB_E_ARG, "unknown field %d", f);
  }
  if (!*ptr) return set_err(ctx, PYIB_E_STATE, "field %d is not allocated", f);
  return PYIB_OK;
}

int pyib_set_field(pyib_ctx* ctx, int32_t field, const void* host, size_t count) {
  if (!ctx || !host) return PYIB_E_ARG;
  void* ptr; size_t n, el; bool wr;
  RET(field_ptr(ctx, field, &ptr, &n, &el, &wr));
  if (!wr || count != n) return set_err(ctx, PYIB_E_ARG, "field %d expects %zu values, got %zu", field, n, count);
  CK(cudaMemcpyAsync(ptr, host, n * el, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (field == PYIB_F_MARKERS) ctx->stencil_valid = false;
  return PYIB_OK;
}

int pyib_get_field(pyib_ctx* ctx, int32_t field, void* host, size_t count) {
  if (!ctx || !host) return PYIB_E_ARG;
  void* ptr; size_t n, el; bool wr;
  RET(field_ptr(ctx, field, &ptr, &n, &el, &wr));
  if (count != n) return set_err(ctx, PYIB_E_ARG, "field %d holds %zu values, asked %zu", field, n, count);
  CK(cudaMemcpyAsync(host, ptr, n * el, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int pyib_matvec(pyib_ctx* ctx, int32_t in_field, int32_t out_field, double dt, int32_t alpd) {
  if (!ctx) return PYIB_E_ARG;
  if (!tables_ready(ctx) || !ctx->have_params) return set_err(ctx, PYIB_E_STATE, "context not ready");
  void *pi, *po; size_t n1, n2, e1, e2; bool w1, w2;
  RET(field_ptr(ctx, in_field, &pi, &n1, &e1, &w1));
  RET(field_ptr(ctx, out_field, &po, &n2, &e2, &w2));
  if (n1 != (size_t)ctx->lay.nedge || n2 != (size_t)ctx->lay.nedge || pi == po)
    return set_err(ctx, PYIB_E_ARG, "matvec needs two distinct edge fields");
  RET(masked_matvec(ctx, (const double*)pi, (double*)po, dt, alpd));
  // zero masked rows (DirBC_s, ib_driver_np.py:32) for the caller
  const long long ne = ctx->lay.nedge;
  k_mask<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, tp<double>(ctx, PYIB_T_PREC), (double*)po);
  CKL();
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int pyib_operator(pyib_ctx* ctx, int32_t op) {
  if (!ctx) return PYIB_E_ARG;
  if (!tables_ready(ctx)) return set_err(ctx, PYIB_E_STATE, "context not ready");
  switch (op) {
    case 0: RET(op_curl(ctx, ctx->work_e, ctx->work_f)); break;
    case 1: RET(op_rot(ctx, ctx->work_f, ctx->work_e)); break;
    case 2: RET(op_interp(ctx, ctx->work_f, ctx->work_c3, ctx->lay.ncell)); break;
    case 3: RET(op_integr(ctx, ctx->work_c3, ctx->lay.ncell, ctx->work_f)); break;
    default: return set_err(ctx, PYIB_E_ARG, "unknown operator %d", op);
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int pyib_calc_vel(pyib_ctx* ctx) {
  if (!ctx) return PYIB_E_ARG;
  if (!tables_ready(ctx)) return set_err(ctx, PYIB_E_STATE, "context not ready");
  RET(op_calc_vel(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int pyib_conv_diff(pyib_ctx* ctx) {
  if (!ctx) return PYIB_E_ARG;
  if (!tables_ready(ctx) || !ctx->have_params) return set_err(ctx, PYIB_E_STATE, "context not ready");
  RET(op_convdiff(ctx, 0, 0, 0, 0, nullptr, nullptr, ctx->work_c3, ctx->res_c));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int pyib_helm_solve(pyib_ctx* ctx, double dt, pyib_solve_stats* stats) {
  if (!ctx) return PYIB_E_ARG;
  if (!tables_ready(ctx) || !ctx->have_params) return set_err(ctx, PYIB_E_STATE, "context not ready");
  return ctx->prm.precision == 1 ? helm_solve_mixed(ctx, dt, stats) : helm_solve(ctx, dt, stats);
}

int pyib_step(pyib_ctx* ctx, double dt, double dt_old, int32_t inner, const double* markers,
              const double* vel, pyib_step_stats* stats) {
  if (!ctx) return PYIB_E_ARG;
  if (!(dt > 0) || !(dt_old > 0)) return set_err(ctx, PYIB_E_ARG, "dt must be positive");
  if ((markers == nullptr) != (vel == nullptr)) return set_err(ctx, PYIB_E_ARG, "markers and vel go together");
  CK(cudaSetDevice(ctx->device));
  return do_step(ctx, dt, dt_old, inner, markers, vel, stats);
}

int pyib_batch_create(pyib_ctx* const* ctxs, int32_t n, pyib_batch** out) {
  if (!ctxs || n < 1 || !out) return PYIB_E_ARG;
  *out = nullptr;
  for (int c = 0; c < n; ++c) {
    if (!ctxs[c]) return PYIB_E_ARG;
    if (ctxs[c]->device != ctxs[0]->device) return set_err(ctxs[c], PYIB_E_ARG, "a batch lives on one device");
    for (int d = 0; d < c; ++d)
      if (ctxs[d] == ctxs[c]) return set_err(ctxs[c], PYIB_E_ARG, "a context appears twice in the batch");
  }
  pyib_batch* b = new pyib_batch();
  b->cs.assign(ctxs, ctxs + n);
  b->device = ctxs[0]->device;
  b->h_cases.assign(n, BCase{});
  auto fail = [&](cudaError_t e) {
    const std::string msg = cudaGetErrorString(e);
    pyib_batch_destroy(b);
    return set_err(ctxs[0], PYIB_E_CUDA, "batch setup failed: %s", msg.c_str());
  };
  cudaError_t e = cudaSetDevice(b->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_cases, n * sizeof(BCase));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int g = 0; g < kBatchGroups && e == cudaSuccess; ++g) {
    e = cudaStreamCreateWithFlags(&b->gstream[g], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[g], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) return fail(e);
  *out = b;
  return PYIB_OK;
}

int pyib_batch_destroy(pyib_batch* b) {
  if (!b) return PYIB_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->d_cases) cudaFree(b->d_cases);
  if (b->d_blk) cudaFree(b->d_blk);
  for (int g = 0; g < kBatchGroups; ++g) {
    if (b->join[g]) cudaEventDestroy(b->join[g]);
    if (b->gstream[g]) cudaStreamDestroy(b->gstream[g]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return PYIB_OK;
}

int pyib_batch_last_error(const pyib_batch* b, char* buf, size_t n) {
  if (!b || !buf || n == 0) return PYIB_E_ARG;
  snprintf(buf, n, "%s", b->err.c_str());
  return PYIB_OK;
}

int pyib_batch_step(pyib_batch* b, const double* dt, const double* dt_old, int32_t inner,
                    const double* const* markers, const double* const* vel, pyib_step_stats* stats) {
  if (!b || !dt || !dt_old) return PYIB_E_ARG;
  b->err.clear();
  const int n = (int)b->cs.size();
  if ((markers == nullptr) != (vel == nullptr)) return batch_err(b, PYIB_E_ARG, "markers and vel go together");
  for (int c = 0; c < n; ++c) {
    const pyib_ctx* ctx = b->cs[c];
    if (!(dt[c] > 0) || !(dt_old[c] > 0)) return batch_err(b, PYIB_E_ARG, "case %d: dt must be positive", c);
    if (markers && ((markers[c] == nullptr) != (vel[c] == nullptr)))
      return batch_err(b, PYIB_E_ARG, "case %d: markers and vel go together", c);
    if (!ctx->have_params) return batch_err(b, PYIB_E_STATE, "case %d: context not ready", c);
    if (ctx->prm.precision != b->cs[0]->prm.precision)
      return batch_err(b, PYIB_E_ARG, "the cases of a batch share one precision");
    if (ctx->prm.check != b->cs[0]->prm.check)
      return batch_err(b, PYIB_E_ARG, "the cases of a batch share one CG check interval");
    if (ctx->use_fused) return batch_err(b, PYIB_E_ARG, "case %d: the single-pass matvec is not batched", c);
  }
  BCK(cudaSetDevice(b->device));
  return batch_step(b, dt, dt_old, inner, markers, vel, stats);
}

int pyib_batch_timing(pyib_batch* b, double* out, int32_t reset) {
  if (!b || !out) return PYIB_E_ARG;
  out[0] = b->chunk_seconds;
  out[1] = (double)b->launches;
  out[2] = (double)b->captures;
  if (reset) {
    b->chunk_seconds = 0.0;
    b->launches = 0;
    b->captures = 0;
  }
  return PYIB_OK;
}

int pyib_ib_stencil(pyib_ctx* ctx) {
  if (!ctx) return PYIB_E_ARG;
  RET(ib_stencil(ctx));
  RET(check_dev_err(ctx));
  return PYIB_OK;
}

int pyib_ib_interp(pyib_ctx* ctx) {
  if (!ctx) return PYIB_E_ARG;
  if (!ctx->stencil_valid) RET(ib_stencil(ctx));
  RET(ib_interp(ctx, ctx->lag));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int pyib_ib_interp_dx(pyib_ctx* ctx, double* jac) {
  if (!ctx || !jac) return PYIB_E_ARG;
  if (ctx->M <= 0) return set_err(ctx, PYIB_E_STATE, "no markers");
  CK(cudaSetDevice(ctx->device));
  if (!ctx->stencil_valid) RET(ib_stencil(ctx));
  k_ib_interp_dx<<<grid_for(ctx->M), kThreads, 0, ctx->stream>>>(
      ctx->M, ncx_of(ctx), ctx->mk, ctx->pos_ref[0], ctx->pos_ref[1], ctx->pos_ref[2], ctx->dx, ctx->prm.hh,
      ctx->prm.hh3, ctx->ib_n[0], ctx->ib_n[1], ctx->ib_n[2], ctx->ibbase, ctx->vc, ctx->ibjac);
  CKL();
  CK(cudaMemcpyAsync(jac, ctx->ibjac, 9 * (size_t)ctx->M * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int pyib_ib_spread(pyib_ctx* ctx) {
  if (!ctx) return PYIB_E_ARG;
  if (!ctx->stencil_valid) RET(ib_stencil(ctx));
  RET(ib_spread(ctx, ctx->fL, ctx->fE));
  CK(cudaStreamSynchronize(ctx->stream));
  return PYIB_OK;
}

int pyib_loads(pyib_ctx* ctx, const double* centre, double radius, double width, double density,
               int32_t fixed_centre, const double* centre0, double* out) {
  if (!ctx || !centre || !out || !centre0) return PYIB_E_ARG;
  if (!ctx->tab[PYIB_T_LC_CAND].ptr || !ctx->tab[PYIB_T_LC_FIDX].ptr || !ctx->tab[PYIB_T_LC_CPOS].ptr)
    return set_err(ctx, PYIB_E_STATE, "load-correction tables missing");
  const double* c = fixed_centre ? centre0 : centre;
  double* dout = ctx->partials + (size_t)(kSlots - 1) * kPartStride;   // 13 doubles of scratch
  const long long n = ctx->n_cand > ctx->n_fidx ? ctx->n_cand : ctx->n_fidx;
  k_loads<<<grid_for(n), kThreads, 0, ctx->stream>>>(
      ctx->n_cand, tp<int>(ctx, PYIB_T_LC_CAND), ctx->n_fidx, tp<int>(ctx, PYIB_T_LC_FIDX),
      tp<double>(ctx, PYIB_T_LC_CPOS), tp<double>(ctx, PYIB_T_VOLCI), ctx->vc, ncx_of(ctx), ctx->fE,
      ctx->lay.ncell, c[0], c[1], c[2], radius, width, ctx->partials, ctx->st, dout);
  CKL();
  double h[13];
  CK(cudaMemcpyAsync(h, dout, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int q = 0; q < 6; ++q) out[q] = h[q];
  for (int q = 6; q < 12; ++q) out[q] = density * h[q];
  out[12] = h[12];
  return PYIB_OK;
}

int pyib_diagnostics(pyib_ctx* ctx, double* out) {
  if (!ctx || !out) return PYIB_E_ARG;
  double* dout = ctx->partials + (size_t)(kSlots - 1) * kPartStride;
  k_diag<<<grid_for(ctx->lay.ncell), kThreads, 0, ctx->stream>>>(
      ctx->lay.ncell, ncx_of(ctx), ctx->vc, tp<long long>(ctx, PYIB_T_CF_PTR), tp<int>(ctx, PYIB_T_CF_FACE),
      tp<double>(ctx, PYIB_T_VOLCI), ctx->U, ctx->partials, ctx->st, dout);
  CKL();
  double h[2];
  CK(cudaMemcpyAsync(h, dout, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  out[0] = h[0];
  out[1] = h[1];
  out[2] = out[3] = 0.0;
  if (ctx->M > 0) {
    if (!ctx->stencil_valid) RET(ib_stencil(ctx));
    RET(ib_interp(ctx, ctx->lag));
    std::vector<double> uL(3 * ctx->M), vel(3 * ctx->M);
    CK(cudaMemcpyAsync(uL.data(), ctx->lag, uL.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(vel.data(), ctx->mvel, vel.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double mx = 0.0, ss = 0.0;
    for (int i = 0; i < ctx->M; ++i) {
      const double a = uL[3 * i] - vel[3 * i], b = uL[3 * i + 1] - vel[3 * i + 1], c = uL[3 * i + 2] - vel[3 * i + 2];
      const double sl = std::sqrt((a * a + b * b) + c * c);
      mx = std::fmax(mx, sl);
      ss += sl * sl;
    }
    out[2] = mx;
    out[3] = std::sqrt(ss / ctx->M);
  }
  return PYIB_OK;
}

int pyib_cg_timing(pyib_ctx* ctx, double* out, int32_t reset) {
  if (!ctx || !out) return PYIB_E_ARG;
  out[0] = ctx->cg_seconds;
  out[1] = (double)ctx->cg_iters;
  out[2] = (double)ctx->launches;
  out[3] = (double)ctx->meta.kz;
  out[4] = (double)ctx->meta.kzR;
  if (reset) {
    ctx->cg_seconds = 0.0;
    ctx->cg_iters = 0;
    ctx->launches = 0;
  }
  return PYIB_OK;
}

int pyib_matvec_plan(pyib_ctx* ctx, int32_t* out) {
  if (!ctx || !out) return PYIB_E_ARG;
  const Meta* ms[2] = {&ctx->meta, &ctx->meta32};
  const bool tuned[2] = {ctx->tuned, ctx->tuned32};
  for (int q = 0; q < 2; ++q) {
    out[4 * q + 0] = tuned[q] ? 1 : 0;
    out[4 * q + 1] = ms[q]->kz;
    out[4 * q + 2] = ms[q]->kzR;
    out[4 * q + 3] = ms[q]->av;
  }
  return PYIB_OK;
}

int pyib_event(pyib_ctx* ctx, int32_t which, double* elapsed_ms) {
  if (!ctx) return PYIB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  if (!ctx->tev0) {
    CK(cudaEventCreate(&ctx->tev0));
    CK(cudaEventCreate(&ctx->tev1));
  }
  if (which == 0) {
    CK(cudaEventRecord(ctx->tev0, ctx->stream));
    return PYIB_OK;
  }
  CK(cudaEventRecord(ctx->tev1, ctx->stream));
  CK(cudaEventSynchronize(ctx->tev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->tev0, ctx->tev1));
  if (elapsed_ms) *elapsed_ms = ms;
  return PYIB_OK;
}

int pyib_graph_pcg(pyib_ctx* ctx, int64_t n, const int64_t* ptr, const int32_t* col, const double* val,
                   const double* rhs, double* x, double rtol, int32_t max_iterations, int32_t* iterations,
                   double* solve_ms) {
  if (!ctx || n <= 0 || !ptr || !col || !val || !rhs || !x || !(rtol > 0.0) || max_iterations <= 0)
    return PYIB_E_ARG;
  CK(cudaSetDevice(ctx->device));
  const long long nnz = ptr[n];
  if (ptr[0] != 0 || nnz <= 0 || nnz >= (1LL << 40)) return set_err(ctx, PYIB_E_ARG, "bad CSR row pointers");
  if (n >= (1LL << 31)) return set_err(ctx, PYIB_E_ARG, "too many rows for int32 columns");
  // every index the device reads is checked here first
  for (long long i = 0; i < n; ++i)
    if (ptr[i + 1] < ptr[i]) return set_err(ctx, PYIB_E_ARG, "CSR row pointers decrease at row %lld", i);
  for (long long k = 0; k < nnz; ++k)
    if (col[k] < 0 || col[k] >= n) return set_err(ctx, PYIB_E_ARG, "CSR column %d out of range at %lld", col[k], k);
  // the matrix and vectors live in the context's grow-only workspace
  long long* dptr; int* dcol; double *dval, *buf, *dparts;
  GState* gs;
  auto carve = [&](Carve& c) {
    dptr = c.take<long long>(n + 1);
    dcol = c.take<int>(nnz);
    dval = c.take<double>(nnz);
    buf = c.take<double>(7 * n);
    dparts = c.take<double>(2 * (size_t)kPartStride);
    gs = c.take<GState>(1);
  };
  Carve size{nullptr};
  carve(size);
  RET(grow(ctx, &ctx->ws, &ctx->ws_bytes, size.off));
  Carve real{(char*)ctx->ws};
  carve(real);
  int rc = [&]() -> int {
    CK(cudaMemsetAsync(gs, 0, sizeof(GState), ctx->stream));
    CK(cudaMemcpyAsync(dptr, ptr, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dcol, col, nnz * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(dval, val, nnz * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    double *b = buf, *dx = buf + n, *r = buf + 2 * n, *z = buf + 3 * n, *p = buf + 4 * n, *q = buf + 5 * n,
           *dinv = buf + 6 * n;
    CK(cudaMemcpyAsync(b, rhs, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    {
      // Jacobi: 1 / diagonal, read from the host CSR
      std::vector<double> dh(n, 0.0);
      for (long long i = 0; i < n; ++i)
        for (long long k = ptr[i]; k < ptr[i + 1]; ++k)
          if (col[k] == i) dh[i] += val[k];
      for (long long i = 0; i < n; ++i) {
        if (!(dh[i] > 0.0)) return set_err(ctx, PYIB_E_ARG, "row %lld has no positive diagonal", i);
        dh[i] = 1.0 / dh[i];
      }
      CK(cudaMemcpyAsync(dinv, dh.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
    }
    GState h{};
    RET(graph_cg(ctx, n, dptr, dcol, dval, b, dinv, dx, r, z, p, q, rtol, max_iterations, dparts, gs, h));
    CK(cudaMemcpyAsync(x, dx, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (solve_ms) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
      *solve_ms = ms;
    }
    const int it = h.iters;
    if (iterations) *iterations = it;
    if (!h.done)
      return set_err(ctx, PYIB_E_NOCONV, "graph PCG did not converge in %d iterations (|r|/|b| = %.3e)", it,
                     std::sqrt(h.rr / (h.bb > 0.0 ? h.bb : 1.0)));
    return PYIB_OK;
  }();
  return rc;
}

int pyib_recover_pressure(pyib_ctx* ctx, int64_t ncell, const double* positions, int64_t nface,
                          const int64_t* face_cells, const double* face_area, const double* gradient, double rtol,
                          int32_t max_iterations, double* pressure, double* info) {
  if (!ctx || !positions || !face_cells || !face_area || !gradient || !pressure || !(rtol > 0.0) ||
      max_iterations <= 0)
    return PYIB_E_ARG;
  if (ncell < 2) return set_err(ctx, PYIB_E_ARG, "pressure recovery needs at least two 3D cells");
  if (ncell >= (1LL << 31) || nface >= (1LL << 30) || nface < 0)
    return set_err(ctx, PYIB_E_ARG, "pressure graph too large (%lld cells, %lld faces)", (long long)ncell,
                   (long long)nface);
  if (nface == 0) return set_err(ctx, PYIB_E_ARG, "pressure graph has no valid internal faces");
  CK(cudaSetDevice(ctx->device));
  const long long n = ncell, nf = nface;
  cudaStream_t st = ctx->stream;
  // every buffer lives in the context's grow-only workspace, sized for the
  // largest key count (two per face)
  double *dpos, *dgrad, *darea, *w_f, *jump_f, *val, *buf, *dparts, *dout;
  long long *dpairs, *ptr;
  unsigned int* deg;
  int *klen, *kptr, *kcur, *col;
  unsigned long long *keys, *keys_sorted;
  unsigned char *bflag, *vis;
  PrState* pst;
  GState* gs;
  auto carve = [&](Carve& c) {
    dpos = c.take<double>(3 * n);
    dgrad = c.take<double>(3 * n);
    darea = c.take<double>(nf);
    dpairs = c.take<long long>(2 * nf);
    w_f = c.take<double>(nf);
    jump_f = c.take<double>(nf);
    deg = c.take<unsigned int>(n);
    klen = c.take<int>(n + 1);
    kptr = c.take<int>(n + 1);
    kcur = c.take<int>(n + 1);
    bflag = c.take<unsigned char>(n);
    vis = c.take<unsigned char>(n);
    pst = c.take<PrState>(1);
    gs = c.take<GState>(1);
    dparts = c.take<double>(3 * (size_t)kPartStride);
    dout = c.take<double>(4);
    buf = c.take<double>(7 * n);
    keys = c.take<unsigned long long>(2 * nf);
    keys_sorted = c.take<unsigned long long>(2 * nf);
    ptr = c.take<long long>(n + 1);
    col = c.take<int>(2 * nf + n);
    val = c.take<double>(2 * nf + n);
  };
  Carve size{nullptr};
  carve(size);
  RET(grow(ctx, &ctx->ws, &ctx->ws_bytes, size.off));
  Carve real{(char*)ctx->ws};
  carve(real);
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  int rc = [&]() -> int {
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaEventRecord(t0, st));
    CK(cudaMemcpyAsync(dpos, positions, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dgrad, gradient, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(darea, face_area, nf * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dpairs, face_cells, 2 * nf * sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(deg, 0, n * sizeof(unsigned int), st));
    CK(cudaMemsetAsync(bflag, 0, n, st));
    CK(cudaMemsetAsync(pst, 0, sizeof(PrState), st));
    CK(cudaMemsetAsync(gs, 0, sizeof(GState), st));
    k_pr_cells<<<grid_for(3 * n), kThreads, 0, st>>>(3 * n, dpos, dgrad, pst);
    CKL();
    k_pr_faces<<<grid_for(nf), kThreads, 0, st>>>(nf, n, dpairs, darea, dpos, dgrad, deg, w_f, jump_f, bflag, pst);
    CKL();
    k_pr_klen<<<grid_for(n + 1), kThreads, 0, st>>>(n, deg, klen);
    CKL();
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, klen, kptr, (int)(n + 1), st));
    RET(grow(ctx, &ctx->ws_tmp, &ctx->ws_tmp_bytes, tb));
    CK(cub::DeviceScan::ExclusiveSum(ctx->ws_tmp, tb, klen, kptr, (int)(n + 1), st));
    PrState hs{};
    int nkeys = 0;
    unsigned int deg0 = 0;
    CK(cudaMemcpyAsync(&hs, pst, sizeof(PrState), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&nkeys, kptr + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&deg0, deg, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // the reference's checks, in its order (ib_postprocess.py:58-79, 88-89)
    if (hs.err & kPrPos) return set_err(ctx, PYIB_E_ARG, "cell_positions contains non-finite values");
    if (hs.err & kPrGrad) return set_err(ctx, PYIB_E_ARG, "gradient contains non-finite values");
    if (hs.err & kPrIds) return set_err(ctx, PYIB_E_ARG, "face_cells contains invalid cell ids");
    if (hs.err & kPrAreaNf) return set_err(ctx, PYIB_E_ARG, "face_area contains non-finite values");
    if (hs.err & kPrAreaNeg) return set_err(ctx, PYIB_E_ARG, "face areas must be positive");
    if ((hs.err & kPrDist) || (long long)nkeys + deg0 == 0)
      return set_err(ctx, PYIB_E_ARG, "pressure graph has no valid internal faces");
    // CSR rows: keys sorted within each row
    const long long nnz = (long long)nkeys + (n - 1);
    CK(cudaMemcpyAsync(kcur, kptr, (n + 1) * sizeof(int), cudaMemcpyDeviceToDevice, st));
    k_pr_fill<<<grid_for(nf), kThreads, 0, st>>>(nf, dpairs, w_f, kcur, keys);
    CKL();
    if (nkeys > 0) {
      size_t sb = 0;
      CK(cub::DeviceSegmentedSort::SortKeys(nullptr, sb, keys, keys_sorted, nkeys, (int)n, kptr, kptr + 1, st));
      RET(grow(ctx, &ctx->ws_tmp, &ctx->ws_tmp_bytes, sb));
      CK(cub::DeviceSegmentedSort::SortKeys(ctx->ws_tmp, sb, keys, keys_sorted, nkeys, (int)n, kptr, kptr + 1, st));
    }
    double *b = buf, *dx = buf + n, *r = buf + 2 * n, *z = buf + 3 * n, *p = buf + 4 * n, *q = buf + 5 * n,
           *dinv = buf + 6 * n;
    k_pr_rows<<<grid_for(n), kThreads, 0, st>>>(n, kptr, keys_sorted, w_f, jump_f, ptr, col, val, b, dinv);
    CKL();
    // connectivity: sweeps until a chunk reaches no new cell (at most n productive sweeps)
    CK(cudaMemsetAsync(vis, 0, n, st));
    CK(cudaMemsetAsync(vis, 1, 1, st));
    unsigned long long seen = 0;
    long long sweeps = 0;
    for (;;) {
      for (int c = 0; c < 8; ++c) {
        k_pr_reach<<<grid_for(n), kThreads, 0, st>>>(n, ptr, col, vis, pst);
        CKL();
      }
      sweeps += 8;
      CK(cudaMemcpyAsync(&hs, pst, sizeof(PrState), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (hs.reached == seen || hs.reached >= (unsigned long long)(n - 1) || sweeps > n + 8) break;
      seen = hs.reached;
    }
    if (hs.reached != (unsigned long long)(n - 1))
      return set_err(ctx, PYIB_E_ARG, "pressure graph is disconnected; a unique gauge is unavailable");
    // the CG (scipy's stop test), from zero
    GState h{};
    RET(graph_cg(ctx, n, ptr, col, val, b, dinv, dx, r, z, p, q, rtol, max_iterations, dparts, gs, h));
    if (!h.done)
      return set_err(ctx, PYIB_E_NOCONV, "pressure graph solve failed to converge (status %d)", max_iterations);
    // gauge: the mean over the cells with a boundary face (every cell if none)
    double g3[3];
    k_pr_gauge<<<grid_for(n), kThreads, 0, st>>>(n, dx, bflag, dparts, &gs->counter, dout);
    CKL();
    CK(cudaMemcpyAsync(g3, dout, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const bool boundary = g3[1] > 0.0;
    const double mean = boundary ? g3[0] / g3[1] : g3[2] / (double)n;
    k_pr_shift<<<grid_for(n), kThreads, 0, st>>>(n, dx, mean);
    CKL();
    double m2[2];
    k_pr_mismatch<<<grid_for(nf), kThreads, 0, st>>>(nf, dpairs, dx, w_f, jump_f, dparts, &gs->counter, dout);
    CKL();
    CK(cudaMemcpyAsync(m2, dout, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(pressure, dx, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(t1, st));
    CK(cudaStreamSynchronize(st));
    if (info) {
      float solve = 0.f, total = 0.f;
      CK(cudaEventElapsedTime(&solve, ctx->ev0, ctx->ev1));
      CK(cudaEventElapsedTime(&total, t0, t1));
      info[0] = std::sqrt(m2[0] / m2[1]);
      info[1] = (double)h.iters;
      info[2] = boundary ? 1.0 : 0.0;
      info[3] = solve;
      info[4] = total;
      info[5] = (double)sweeps;
      info[6] = (double)nnz;
    }
    return PYIB_OK;
  }();
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  return rc;
}

int pyib_bench_matvec(pyib_ctx* ctx, int32_t reps, double dt, double* ms_per) {
  if (!ctx || reps <= 0 || !ms_per) return PYIB_E_ARG;
  if (!tables_ready(ctx) || !ctx->have_params) return set_err(ctx, PYIB_E_STATE, "context not ready");
  CK(cudaSetDevice(ctx->device));
  RET(tune_matvec(ctx));
  RET(set_state_solver(ctx, dt, 1));
  if (ctx->prm.precision == 1) {
    // the float32 matvec of the mixed solver, on a float32 copy of WORK_E
    RET(ensure_mixed(ctx));
    RET(tune_matvec32(ctx));
    const long long ne = ctx->lay.nedge;
    k_d2f<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->work_e, ctx->p32);
    CKL();
    return bench_matvec_t<float>(ctx, reps, ctx->p32, ctx->w32, ctx->vcm32, ctx->vq32, ctx->pa_val32,
                                 ctx->pv_val32, ctx->pr_val32, ms_per);
  }
  return bench_matvec_t<double>(ctx, reps, ctx->work_e, ctx->work_e2, ctx->vcm, ctx->vq,
                                tp<double>(ctx, PYIB_T_PA_VAL), tp<double>(ctx, PYIB_T_PV_VAL),
                                tp<double>(ctx, PYIB_T_PR_VAL), ms_per);
}

// The fused float64 matvec timed with CUDA events: ms_per[0] the whole matvec,
// [1] the exact vc rows and listed template vc, [2] the exact vq rows, [3] k_mvF,
// [4] the exact w rows with the final dot.
int pyib_bench_matvec_fused(pyib_ctx* ctx, int32_t reps, double dt, double* ms_per) {
  if (!ctx || !ms_per || reps <= 0) return PYIB_E_ARG;
  if (!tables_ready(ctx) || !ctx->have_params) return set_err(ctx, PYIB_E_STATE, "context not ready");
  CK(cudaSetDevice(ctx->device));
  RET(set_state_solver(ctx, dt, 1));
  RET(tune_fused(ctx));
  RET(set_state_solver(ctx, dt, 1));
  const double* in = ctx->work_e;
  double* out = ctx->work_e2;
  RET(launch_matvec_fused(ctx, in, out, 1));   // warm
  float ms = 0.f;
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  for (int q = 0; q < reps; ++q) RET(launch_matvec_fused(ctx, in, out, 1));
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaEventSynchronize(ctx->ev1));
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ms_per[0] = ms / reps;
  const Meta& m = ctx->meta;
  const long long nc = ctx->lay.ncell;
  const FusedTabs tb{ctx->f_irrA, ctx->f_irrV, ctx->f_needR, tp<unsigned int>(ctx, PYIB_T_PR_BITS),
                     ctx->f_flags};
  for (int kern = 0; kern < 4; ++kern) {
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    for (int q = 0; q < reps; ++q) {
      if (kern == 0) {
        if (ctx->nA > 0) {
          k_patchA<double><<<patch_grid(3 * ctx->nA), kThreads, 0, ctx->stream>>>(
              ctx->nA, tp<int>(ctx, PYIB_T_PA_IDS), tp<long long>(ctx, PYIB_T_PA_PTR),
              tp<int>(ctx, PYIB_T_PA_COL), tp<double>(ctx, PYIB_T_PA_VAL), in, ctx->vcm, nc, ctx->st);
          CKL();
        }
        if (ctx->n_list > 0) {
          k_vc_list<<<patch_grid(ctx->n_list), kThreads, 0, ctx->stream>>>(m, ctx->n_list, ctx->f_list, in,
                                                                            ctx->vcm, ctx->st);
          CKL();
        }
      } else if (kern == 1) {
        if (ctx->nV > 0) {
          k_patchV<double><<<patch_grid(ctx->nV), kThreads, 0, ctx->stream>>>(
              ctx->nV, tp<int>(ctx, PYIB_T_PV_IDS), tp<long long>(ctx, PYIB_T_PV_PTR),
              tp<int>(ctx, PYIB_T_PV_COL), tp<double>(ctx, PYIB_T_PV_VAL), ctx->vcm, ctx->vq, nc, ctx->st);
          CKL();
        }
      } else if (kern == 2) {
        k_mvF<<<dim3(m.gxF, m.gyF, m.gzF), dim3(FX, FY, 1), kFusedSmemBytes, ctx->stream>>>(m, in, out, ctx->vcm, ctx->vq, tb,
                                                                             ctx->partials, ctx->st, 1);
        CKL();
      } else {
        k_patchRI<double><<<patch_grid(ctx->nR), kThreads, 0, ctx->stream>>>(
            ctx->nR, tp<int>(ctx, PYIB_T_PR_IDS), tp<long long>(ctx, PYIB_T_PR_PTR), tp<int>(ctx, PYIB_T_PR_COL),
            tp<double>(ctx, PYIB_T_PR_VAL), ctx->vq, out, in, ctx->partials, m.nplanesF, ctx->st, 1);
        CKL();
      }
    }
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ms_per[1 + kern] = ms / reps;
  }
  ms_per[5] = (double)m.kzF;
  return PYIB_OK;
}

}  // extern "C"

// ===========================================================================
// Spreading without allocation.
//
// Some callers cannot call cudaMalloc: a coupling code that runs inside a
// memory budget fixed at start-up, or a host framework whose allocator owns
// all device memory, still needs the deterministic spreading of Lagrangian
// forces.  pyib_spread_noalloc keeps all its scratch (sort keys and values in
// two ping-pong pairs, and CUB's temporary storage) in one file-scope
// __device__ array of fixed size; every GPU that loads this library holds it
// until the process exits.  The caller passes inputs and the output.
// ===========================================================================
namespace {
constexpr long long kNoAllocMaxMarkers = 8192;                      // 1,024,000 contributions
constexpr long long kNoAllocMaxItems = kNoAllocMaxMarkers * 125;
constexpr size_t kNoAllocSortBytes = 4ull * kNoAllocMaxItems * sizeof(int);   // 16,384,000
constexpr size_t kNoAllocTempBytes = 1ull << 20;                   // CUB histograms and offsets
constexpr size_t kNoAllocStatusBytes = 256;                        // reject counter
constexpr size_t kNoAllocBytes = kNoAllocSortBytes + kNoAllocTempBytes + kNoAllocStatusBytes;
constexpr int kNoAllocMaxDevices = 64;
}  // namespace

static __device__ __align__(256) unsigned char g_spread_scratch[kNoAllocBytes];
static void* g_spread_scratch_ptr[kNoAllocMaxDevices] = {nullptr};

namespace {
// Keys for the no-allocation spreading: caller-supplied cell ids are checked
// against [0, ncell).  A bad id gets the sentinel key ncell, which sorts after
// every valid cell and which k_ib_segsum skips, so it writes nothing; the
// rejects are counted in a word of the fixed scratch array.
__global__ void k_noalloc_keys(long long tot, long long ncell, const int* __restrict__ cell, int* keys,
                               int* vals, unsigned int* rejects) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = cell[t];
    const bool ok = c >= 0 && (long long)c < ncell;
    keys[t] = ok ? c : (int)ncell;
    vals[t] = (int)t;
    if (!ok) atomicAdd(rejects, 1u);
  }
}
}  // namespace

extern "C" int pyib_spread_noalloc(const int32_t* cell, const double* w, const double* ds3, const double* f,
                                   int32_t nmarkers, int64_t ncell, double* out, void* stream) {
  if (!cell || !w || !ds3 || !f || !out) return PYIB_E_ARG;
  if (nmarkers <= 0 || nmarkers > kNoAllocMaxMarkers) return PYIB_E_ARG;
  if (ncell <= 0 || ncell >= (1LL << 31)) return PYIB_E_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PYIB_E_CUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return PYIB_E_ARG;
  if (!g_spread_scratch_ptr[dev]) {
    // Host code only sees a stand-in for the array; the kernels need its device address.
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_spread_scratch) != cudaSuccess || !p) return PYIB_E_CUDA;
    g_spread_scratch_ptr[dev] = p;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const long long tot = (long long)nmarkers * 125;
  int* keys_a = (int*)g_spread_scratch_ptr[dev];
  int* keys_b = keys_a + kNoAllocMaxItems;
  int* vals_a = keys_b + kNoAllocMaxItems;
  int* vals_b = vals_a + kNoAllocMaxItems;
  void* temp = (void*)((unsigned char*)g_spread_scratch_ptr[dev] + kNoAllocSortBytes);
  unsigned int* rejects =
      (unsigned int*)((unsigned char*)g_spread_scratch_ptr[dev] + kNoAllocSortBytes + kNoAllocTempBytes);
  // enough key bits for every valid id and the sentinel ncell (ncell < 2^31)
  int nbits = 1;
  while (nbits < 31 && (1LL << nbits) <= ncell) ++nbits;
  cub::DoubleBuffer<int> dk(keys_a, keys_b), dv(vals_a, vals_b);
  size_t tb = 0;
  if (cub::DeviceRadixSort::SortPairs((void*)nullptr, tb, dk, dv, (int)tot, 0, nbits, s) != cudaSuccess)
    return PYIB_E_CUDA;
  if (tb > kNoAllocTempBytes) return PYIB_E_ARG;
  if (cudaMemsetAsync(out, 0, 3 * (size_t)ncell * sizeof(double), s) != cudaSuccess) return PYIB_E_CUDA;
  // the array keeps the previous call's contents: the reject count starts at zero
  if (cudaMemsetAsync(rejects, 0, sizeof(unsigned int), s) != cudaSuccess) return PYIB_E_CUDA;
  k_noalloc_keys<<<grid_for(tot), kThreads, 0, s>>>(tot, ncell, cell, dk.Current(), dv.Current(), rejects);
  if (cudaGetLastError() != cudaSuccess) return PYIB_E_CUDA;
  if (cub::DeviceRadixSort::SortPairs(temp, tb, dk, dv, (int)tot, 0, nbits, s) != cudaSuccess)
    return PYIB_E_CUDA;
  k_ib_segsum<<<grid_for(tot), kThreads, 0, s>>>(tot, ncell, dk.Current(), dv.Current(), w, ds3, f, out);
  if (cudaGetLastError() != cudaSuccess) return PYIB_E_CUDA;
  // Stream-ordered read of the reject count: the call returns once its work is done.
  unsigned int bad = 0;
  if (cudaMemcpyAsync(&bad, rejects, sizeof(bad), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PYIB_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return PYIB_E_CUDA;
  return bad ? PYIB_E_DEVICE : PYIB_OK;
}
