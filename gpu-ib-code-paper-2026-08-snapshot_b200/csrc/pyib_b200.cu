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

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pyib_b200.h"

#define PYIB_VERSION "pyib_b200 0.1.0 sm_100a"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 8;      // fixed reduction grid (148 SMs x 8)
constexpr int kSlots = 16;               // reduction values per block

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
};

struct Meta {
  int nl;
  LevelMeta lv[PYIB_MAX_LEVELS];
  long long nc, nf, ne;
};

struct CGState {
  double eta, eta_new, pw, alpha, beta, thresh, l2_0, xnorm;
  double true_eta, true_l2, tol1, tol2;
  double rou, kfac;              // V block: rou*v - kfac*(Vd v)
  int m, done, iters, check, cg_max, alpd, pad0, pad1;
  unsigned int counter;
  unsigned int pad2;
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
  // reduction / state
  double* partials = nullptr;
  CGState* st = nullptr;
  CGState* st_host = nullptr;     // pinned
  // IB
  int M = 0;
  double *mk = nullptr, *mvel = nullptr, *ds = nullptr, *fL = nullptr, *lag = nullptr,
         *dL = nullptr, *ibw = nullptr;
  int *ibcell = nullptr, *ibbase = nullptr;
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
  int cg_graph_alpd = -1;
  // timing
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, tev0 = nullptr, tev1 = nullptr;
  double cg_seconds = 0.0;
  long long cg_iters = 0;
  long long launches = 0;        // kernels launched by this context
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

// ---------------------------------------------------------------------------
// deterministic block reduction
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh /*[NV*32]*/) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double t = v[q];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[q * 32 + wid] = t;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double t = lane < nw ? sh[q * 32 + lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      v[q] = t;
    }
  }
  __syncthreads();
}

// Writes this block's partials; returns true in the block that finishes last,
// whose thread 0 then holds the totals in v (summed in block order).
template <int NV>
__device__ bool grid_sum(double (&v)[NV], double* partials, unsigned int* counter) {
  __shared__ double sh[NV * 32];
  __shared__ bool last;
  block_sum<NV>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[q * kMaxBlocks + blockIdx.x] = v[q];
    __threadfence();
    unsigned int t = atomicAdd(counter, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double t = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
      t += ((volatile double*)partials)[q * kMaxBlocks + b];
    acc[q] = t;
  }
  block_sum<NV>(acc, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = acc[q];
    *counter = 0u;
  }
  return true;
}

// ---------------------------------------------------------------------------
// layout decoding
// ---------------------------------------------------------------------------
__device__ __forceinline__ int level_of_cell(const Meta& m, long long c) {
  int L = 0;
  while (L + 1 < m.nl && c >= m.lv[L + 1].cbase) ++L;
  return L;
}

__device__ __forceinline__ bool in_hole(const LevelMeta& l, int i, int j, int k) {
  return l.has_hole && i >= l.hole_lo[0] && i < l.hole_hi[0] && j >= l.hole_lo[1] &&
         j < l.hole_hi[1] && k >= l.hole_lo[2] && k < l.hole_hi[2];
}

__device__ __forceinline__ bool bit_set(const unsigned int* bits, long long i) {
  return (bits[i >> 5] >> (i & 31)) & 1u;
}

// ---------------------------------------------------------------------------
// matvec kernel A: vc = P C p (template + patch)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_mvA(Meta m, const T* __restrict__ p, T* __restrict__ vc,
                                                  const unsigned int* __restrict__ pbits,
                                                  const int* __restrict__ prow,
                                                  const long long* __restrict__ pptr,
                                                  const int* __restrict__ pcol,
                                                  const T* __restrict__ pval, long long nA,
                                                  const CGState* __restrict__ st) {
  if (st && st->done) return;
  const long long nc = m.nc;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc;
       c += (long long)gridDim.x * blockDim.x) {
    const int L = level_of_cell(m, c);
    const LevelMeta& l = m.lv[L];
    const int nx = l.n[0], ny = l.n[1];
    int loc = (int)(c - l.cbase);
    const int i = loc % nx, j = (loc / nx) % ny, k = loc / (nx * ny);
    if (in_hole(l, i, j, k)) continue;
    if (pbits && bit_set(pbits, c)) {
      const int r = prow[c];
      for (int d = 0; d < 3; ++d) {
        T acc = 0;
        const long long rr = r + d * nA;
        for (long long q = pptr[rr]; q < pptr[rr + 1]; ++q) acc += pval[q] * p[pcol[q]];
        vc[d * nc + c] = acc;
      }
      continue;
    }
    const T* ex = p + l.ebase[0];
    const T* ey = p + l.ebase[1];
    const T* ez = p + l.ebase[2];
    // x-edges dims (nx, ny+1, nz+1); y-edges (nx+1, ny, nz+1); z-edges (nx+1, ny+1, nz)
    auto EX = [&](int a, int b, int cc) { return ex[((long long)cc * (ny + 1) + b) * nx + a]; };
    auto EY = [&](int a, int b, int cc) { return ey[((long long)cc * ny + b) * (nx + 1) + a]; };
    auto EZ = [&](int a, int b, int cc) { return ez[((long long)cc * (ny + 1) + b) * (nx + 1) + a]; };
    const T ex00 = EX(i, j, k), ex10 = EX(i, j + 1, k), ex01 = EX(i, j, k + 1), ex11 = EX(i, j + 1, k + 1);
    const T ey00 = EY(i, j, k), ey10 = EY(i + 1, j, k), ey01 = EY(i, j, k + 1), ey11 = EY(i + 1, j, k + 1);
    const T ez00 = EZ(i, j, k), ez10 = EZ(i + 1, j, k), ez01 = EZ(i, j + 1, k), ez11 = EZ(i + 1, j + 1, k);
    const T ux0 = ey00 + ez01 - ey01 - ez00;
    const T ux1 = ey10 + ez11 - ey11 - ez10;
    const T uy0 = ez00 + ex01 - ez10 - ex00;
    const T uy1 = ez01 + ex11 - ez11 - ex10;
    const T uz0 = ex00 + ey10 - ex10 - ey00;
    const T uz1 = ex01 + ey11 - ex11 - ey01;
    const T s = (T)(1.0 / (2.0 * l.h * l.h));
    vc[c] = (ux0 + ux1) * s;
    vc[nc + c] = (uy0 + uy1) * s;
    vc[2 * nc + c] = (uz0 + uz1) * s;
  }
}

// ---------------------------------------------------------------------------
// matvec kernel V: vq = rou v - kfac * Vd v  (per component; template + patch)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_mvV(Meta m, const T* __restrict__ v, T* __restrict__ vq,
                                                  const unsigned int* __restrict__ pbits,
                                                  const int* __restrict__ prow,
                                                  const long long* __restrict__ pptr,
                                                  const int* __restrict__ pcol,
                                                  const T* __restrict__ pval,
                                                  const CGState* __restrict__ st) {
  if (st->done) return;
  const long long nc = m.nc;
  const T rou = (T)st->rou, kf = (T)st->kfac;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc;
       c += (long long)gridDim.x * blockDim.x) {
    const int L = level_of_cell(m, c);
    const LevelMeta& l = m.lv[L];
    const int nx = l.n[0], ny = l.n[1], nz = l.n[2];
    int loc = (int)(c - l.cbase);
    const int i = loc % nx, j = (loc / nx) % ny, k = loc / (nx * ny);
    if (in_hole(l, i, j, k)) continue;
    if (pbits && bit_set(pbits, c)) {
      const int r = prow[c];
      for (int d = 0; d < 3; ++d) {
        T acc = 0;
        const T* vd = v + d * nc;
        for (long long q = pptr[r]; q < pptr[r + 1]; ++q) acc += pval[q] * vd[pcol[q]];
        vq[d * nc + c] = rou * vd[c] - kf * acc;
      }
      continue;
    }
    const T inv_h2 = (T)(1.0 / (l.h * l.h));
    const long long sx = 1, sy = nx, sz = (long long)nx * ny;
    for (int d = 0; d < 3; ++d) {
      const T* vd = v + d * nc;
      const T vc0 = vd[c];
      T acc = 0;
      acc += (i + 1 < nx) ? vd[c + sx] - vc0 : -2 * vc0;
      acc += (i > 0) ? vd[c - sx] - vc0 : -2 * vc0;
      acc += (j + 1 < ny) ? vd[c + sy] - vc0 : -2 * vc0;
      acc += (j > 0) ? vd[c - sy] - vc0 : -2 * vc0;
      acc += (k + 1 < nz) ? vd[c + sz] - vc0 : -2 * vc0;
      acc += (k > 0) ? vd[c - sz] - vc0 : -2 * vc0;
      vq[d * nc + c] = rou * vc0 - kf * (acc * inv_h2);
    }
  }
}

// ---------------------------------------------------------------------------
// matvec kernel RI: w = R I vq (template + patch), fused dot p.w, alpha
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T face_F(const LevelMeta& l, const T* __restrict__ vq, long long nc, int a,
                                    int fi, int fj, int fk) {
  // F on the a-face at (fi,fj,fk): (h/2)(vq_a[lo cell] + vq_a[hi cell]); zero outside the box
  if (fi < 0 || fj < 0 || fk < 0) return 0;
  if (fi >= l.n[0] + (a == 0) || fj >= l.n[1] + (a == 1) || fk >= l.n[2] + (a == 2)) return 0;
  const T* va = vq + a * nc + l.cbase;
  const long long sy = l.n[0], sz = (long long)l.n[0] * l.n[1];
  const int fa = a == 0 ? fi : (a == 1 ? fj : fk);
  const long long off = fk * sz + fj * sy + fi;
  const long long sa = a == 0 ? 1 : (a == 1 ? sy : sz);
  T s = 0;
  if (fa > 0) s += va[off - sa];          // lo cell = f - e_a
  if (fa < l.n[a]) s += va[off];          // hi cell = f
  return (T)(0.5 * l.h) * s;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_mvRI(Meta m, const T* __restrict__ vq, T* __restrict__ w,
                                                   const T* __restrict__ p,
                                                   const unsigned int* __restrict__ pbits,
                                                   const int* __restrict__ prow,
                                                   const long long* __restrict__ pptr,
                                                   const int* __restrict__ pcol,
                                                   const T* __restrict__ pval, double* partials,
                                                   CGState* st, int do_dot) {
  if (st->done) return;
  const long long ne = m.ne, nc = m.nc;
  double dot[1] = {0.0};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    T val;
    if (pbits && bit_set(pbits, e)) {
      const int r = prow[e];
      T acc = 0;
      for (long long q = pptr[r]; q < pptr[r + 1]; ++q) acc += pval[q] * vq[pcol[q]];
      val = acc;
    } else {
      int L = 0, t = 0;
      for (;;) {
        const LevelMeta& l = m.lv[L];
        if (e < l.ebase[2] + l.ecount[2]) {
          t = e >= l.ebase[2] ? 2 : (e >= l.ebase[1] ? 1 : 0);
          break;
        }
        ++L;
      }
      const LevelMeta& l = m.lv[L];
      const int dx = l.n[0] + (t != 0), dy = l.n[1] + (t != 1);
      const int loc = (int)(e - l.ebase[t]);
      const int i = loc % dx, j = (loc / dx) % dy, k = loc / (dx * dy);
      const int t1 = (t + 1) % 3, t2 = (t + 2) % 3;
      int q1[3] = {i, j, k}, q2[3] = {i, j, k};
      q1[t1] -= 1;   // idx - e_{t+1}
      q2[t2] -= 1;   // idx - e_{t+2}
      val = face_F<T>(l, vq, nc, t2, i, j, k) - face_F<T>(l, vq, nc, t2, q1[0], q1[1], q1[2]) +
            face_F<T>(l, vq, nc, t1, q2[0], q2[1], q2[2]) - face_F<T>(l, vq, nc, t1, i, j, k);
    }
    w[e] = val;
    if (do_dot) dot[0] += (double)p[e] * (double)val;
  }
  if (!do_dot) return;
  if (grid_sum<1>(dot, partials, &st->counter) && threadIdx.x == 0) {
    st->pw = dot[0];
    st->alpha = st->eta / (dot[0] != 0.0 ? dot[0] : INFINITY);
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
  }
}

__global__ void __launch_bounds__(kThreads) k_cg_update(long long ne, double* x, double* r,
                                                        const double* __restrict__ p,
                                                        const double* __restrict__ w,
                                                        const double* __restrict__ prec,
                                                        double* partials, CGState* st) {
  if (st->done) return;
  const double alpha = st->alpha;
  double v[1] = {0.0};
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x) {
    const double pr = prec[e];
    x[e] += alpha * p[e];
    if (pr != 0.0) {
      const double re = r[e] - alpha * w[e];
      r[e] = re;
      v[0] += (re * pr) * re;
    }
  }
  if (grid_sum<1>(v, partials, &st->counter) && threadIdx.x == 0) {
    const double en = v[0];
    st->eta_new = en;
    const int m = st->m + 1;
    st->m = m;
    bool stop = false;
    if (m % st->check == 0) {
      if (!isfinite(en) || en < st->thresh) stop = true;
    }
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

__global__ void __launch_bounds__(kThreads) k_cg_p(long long ne, const double* __restrict__ r,
                                                   const double* __restrict__ prec, double* p,
                                                   const CGState* st) {
  if (st->done) return;
  const double beta = st->beta;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne;
       e += (long long)gridDim.x * blockDim.x)
    p[e] = r[e] * prec[e] + beta * p[e];
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
    partials[kMaxBlocks + blockIdx.x] = dmax;
    __threadfence();
    unsigned int t = atomicAdd(&st->counter, 1u);
    if (t == gridDim.x - 1) {
      __threadfence();
      double a = 0.0, b = 0.0;
      for (int q = 0; q < (int)gridDim.x; ++q) {
        a = fmax(a, ((volatile double*)partials)[q]);
        b = fmax(b, ((volatile double*)partials)[kMaxBlocks + q]);
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
    case PYIB_T_LC_CPOS:
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
  const int need[] = {PYIB_T_PREC, PYIB_T_CURL_PTR, PYIB_T_ROT_PTR, PYIB_T_P_PTR, PYIB_T_I_PTR,
                      PYIB_T_CF_PTR, PYIB_T_F_LO, PYIB_T_F_HI, PYIB_T_F_AOL, PYIB_T_VOLCI};
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
int launch_matvec(pyib_ctx* ctx, const double* in, double* out, int alpd, int do_dot) {
  const long long nc = ctx->lay.ncell, ne = ctx->lay.nedge;
  k_mvA<double><<<grid_for(nc), kThreads, 0, ctx->stream>>>(
      ctx->meta, in, ctx->vcm, tp<unsigned int>(ctx, PYIB_T_PA_BITS), tp<int>(ctx, PYIB_T_PA_ROW),
      tp<long long>(ctx, PYIB_T_PA_PTR), tp<int>(ctx, PYIB_T_PA_COL), tp<double>(ctx, PYIB_T_PA_VAL),
      ctx->nA, ctx->st);
  CKL();
  const double* vsrc = ctx->vcm;
  if (alpd) {
    k_mvV<double><<<grid_for(nc), kThreads, 0, ctx->stream>>>(
        ctx->meta, ctx->vcm, ctx->vq, tp<unsigned int>(ctx, PYIB_T_PV_BITS), tp<int>(ctx, PYIB_T_PV_ROW),
        tp<long long>(ctx, PYIB_T_PV_PTR), tp<int>(ctx, PYIB_T_PV_COL), tp<double>(ctx, PYIB_T_PV_VAL),
        ctx->st);
    CKL();
    vsrc = ctx->vq;
  }
  k_mvRI<double><<<grid_for(ne), kThreads, 0, ctx->stream>>>(
      ctx->meta, vsrc, out, ctx->p, tp<unsigned int>(ctx, PYIB_T_PR_BITS), tp<int>(ctx, PYIB_T_PR_ROW),
      tp<long long>(ctx, PYIB_T_PR_PTR), tp<int>(ctx, PYIB_T_PR_COL), tp<double>(ctx, PYIB_T_PR_VAL),
      ctx->partials, ctx->st, do_dot);
  CKL();
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
  h.counter = 0u;
  CK(cudaMemcpyAsync(ctx->st, &h, sizeof(CGState), cudaMemcpyHostToDevice, ctx->stream));
  return PYIB_OK;
}

int masked_matvec(pyib_ctx* ctx, const double* in, double* out, double dt, int alpd) {
  RET(set_state_solver(ctx, dt, alpd));
  RET(launch_matvec(ctx, in, out, alpd, 0));
  return PYIB_OK;
}

// one CG iteration (5 kernels)
int cg_iteration(pyib_ctx* ctx) {
  RET(launch_matvec(ctx, ctx->p, ctx->w, 1, 1));
  const long long ne = ctx->lay.nedge;
  k_cg_update<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->x, ctx->r, ctx->p, ctx->w,
                                                          tp<double>(ctx, PYIB_T_PREC), ctx->partials,
                                                          ctx->st);
  CKL();
  k_cg_p<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->r, tp<double>(ctx, PYIB_T_PREC), ctx->p,
                                                     ctx->st);
  CKL();
  return PYIB_OK;
}

int build_cg_graph(pyib_ctx* ctx) {
  if (ctx->cg_graph && ctx->cg_graph_check == ctx->prm.check) return PYIB_OK;
  if (ctx->cg_graph) {
    cudaGraphExecDestroy(ctx->cg_graph);
    ctx->cg_graph = nullptr;
  }
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int rc = PYIB_OK;
  for (int q = 0; q < ctx->prm.check && rc == PYIB_OK; ++q) rc = cg_iteration(ctx);
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (rc != PYIB_OK) return rc;
  if (e != cudaSuccess) return set_err(ctx, PYIB_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&ctx->cg_graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return set_err(ctx, PYIB_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
  ctx->cg_graph_check = ctx->prm.check;
  return PYIB_OK;
}

// PCG from warm start s with right-hand side residual res_e (ib_driver_np.py:311-410).
int helm_solve(pyib_ctx* ctx, double dt, pyib_solve_stats* out) {
  const long long ne = ctx->lay.nedge;
  const double* prec = tp<double>(ctx, PYIB_T_PREC);
  RET(set_state_solver(ctx, dt, 1));
  RET(build_cg_graph(ctx));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  k_cg_init<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->res_e, ctx->s, prec, ctx->x, ctx->r,
                                                        ctx->p, ctx->partials, ctx->st);
  CKL();
  CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const bool start_converged = ctx->st_host->eta < ctx->st_host->thresh;
  int iters = 0;
  if (!start_converged) {
    const long long max_chunks = (ctx->prm.cg_max + ctx->prm.check - 1) / ctx->prm.check + 1;
    for (long long q = 0; q < max_chunks; ++q) {
      CK(cudaGraphLaunch(ctx->cg_graph, ctx->stream));
      ctx->launches += 5LL * ctx->prm.check;
      CK(cudaMemcpyAsync(ctx->st_host, ctx->st, sizeof(CGState), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      if (ctx->st_host->done) break;
    }
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

int ib_alloc(pyib_ctx* ctx, int M) {
  if (ctx->M == M && ctx->mk) return PYIB_OK;
  void* ptrs[] = {ctx->mk, ctx->mvel, ctx->ds, ctx->fL, ctx->lag, ctx->dL, ctx->ibw, ctx->ibcell,
                  ctx->ibbase, ctx->sort_keys_in, ctx->sort_keys_out, ctx->sort_vals_in,
                  ctx->sort_vals_out, ctx->sort_tmp};
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
int do_step(pyib_ctx* ctx, double dt, double dt_old, int inner, const double* markers,
            const double* vel, pyib_step_stats* out) {
  if (!tables_ready(ctx) || !ctx->have_params) return set_err(ctx, PYIB_E_STATE, "context not ready");
  if (inner < 2) return set_err(ctx, PYIB_E_ARG, "accumulated_explicit requires at least 2 fluid inner iterations");
  const pyib_params& P = ctx->prm;
  const long long nc = ctx->lay.ncell, ne = ctx->lay.nedge;
  const bool ib = ctx->M > 0;
  pyib_step_stats st{};
  st.all_converged = 1;
  if (ib && markers) {
    CK(cudaMemcpyAsync(ctx->mk, markers, 3 * ctx->M * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->mvel, vel, 3 * ctx->M * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    RET(ib_stencil(ctx));
    RET(ib_spread(ctx, ctx->fL, ctx->fE));        // held force follows the body (ib_driver_np.py:447-451)
  } else if (ib && !ctx->stencil_valid) {
    RET(ib_stencil(ctx));
  }
  RET(op_calc_vel(ctx));
  const double rou = P.rou, ac = P.ac, ad = P.ad;
  RET(op_convdiff(ctx, 1, ((1.0 - ac) * dt) * rou, (1.0 - ad) * dt, dt, nullptr, nullptr, ctx->res_c0, nullptr));
  k_guess<<<grid_for(ne), kThreads, 0, ctx->stream>>>(ne, ctx->s, ctx->s_old, ctx->prev, dt, dt_old);
  CKL();
  RET(op_calc_vel(ctx));
  for (int it = 1; it <= inner; ++it) {
    RET(op_convdiff(ctx, 2, (ac * dt) * rou, ad * dt, dt, ctx->res_c0, ib ? ctx->fE : nullptr, ctx->res_c,
                    nullptr));
    RET(op_integr(ctx, ctx->res_c, nc, ctx->F));
    RET(op_rot(ctx, ctx->F, ctx->res_e));
    pyib_solve_stats ss{};
    int rc = helm_solve(ctx, dt, &ss);
    st.max_iterations = ss.iterations > st.max_iterations ? ss.iterations : st.max_iterations;
    st.total_iterations += ss.iterations;
    st.max_rel_residual = fmax(st.max_rel_residual, ss.rel_residual);
    st.max_tol_ratio = fmax(st.max_tol_ratio, ss.tol_ratio);
    st.all_converged = st.all_converged && ss.converged;
    if (out) *out = st;
    if (rc != PYIB_OK) return rc;
    RET(op_calc_vel(ctx));
    if (ib && it == 1) {
      RET(ib_interp(ctx, ctx->lag));
      k_ib_force<<<grid_for(3 * ctx->M), kThreads, 0, ctx->stream>>>(ctx->M, ctx->mvel, ctx->lag, dt, ctx->dL);
      CKL();
      RET(ib_spread(ctx, ctx->dL, ctx->conv));   // conv is free scratch here
      k_axpy_scaled<<<grid_for(3 * nc), kThreads, 0, ctx->stream>>>(3 * nc, ctx->fE, rou, ctx->conv);
      CKL();
      k_axpy_scaled<<<grid_for(3 * ctx->M), kThreads, 0, ctx->stream>>>(3 * ctx->M, ctx->fL, rou, ctx->dL);
      CKL();
      st.ib_updates += 1;
    }
  }
  RET(check_dev_err(ctx));
  if (out) *out = st;
  return PYIB_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
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
    RET(alloc(ctx, (void**)&ctx->partials, kSlots * kMaxBlocks * sizeof(double)));
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
  for (auto& t : ctx->tab)
    if (t.ptr) cudaFree(t.ptr);
  void* ptrs[] = {ctx->s, ctx->s_old, ctx->U, ctx->vc, ctx->res_c0, ctx->res_c, ctx->res_e, ctx->F,
                  ctx->fE, ctx->conv, ctx->diff, ctx->work_e, ctx->work_e2, ctx->work_c3, ctx->work_f,
                  ctx->x, ctx->r, ctx->p, ctx->w, ctx->vcm, ctx->vq, ctx->prev, ctx->partials, ctx->st,
                  ctx->dev_err, ctx->mk, ctx->mvel, ctx->ds, ctx->fL, ctx->lag, ctx->dL, ctx->ibw,
                  ctx->ibcell, ctx->ibbase, ctx->sort_keys_in, ctx->sort_keys_out, ctx->sort_vals_in,
                  ctx->sort_vals_out, ctx->sort_tmp, ctx->x32, ctx->r32, ctx->p32, ctx->w32,
                  ctx->vcm32, ctx->vq32, ctx->prec32};
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
  if (table == PYIB_T_INLET_IDX) ctx->n_inlet = bytes / 4;
  if (table == PYIB_T_BF_FACE) ctx->n_bf = bytes / 4;
  if (table == PYIB_T_LC_CAND) ctx->n_cand = bytes / 4;
  if (table == PYIB_T_LC_FIDX) ctx->n_fidx = bytes / 4;
  ctx->cg_graph_check = -1;  // tables changed: recapture
  return PYIB_OK;
}

int pyib_finalize(pyib_ctx* ctx, const int64_t* counts, int32_t ncounts) {
  if (!ctx || !counts || ncounts < 3) return PYIB_E_ARG;
  ctx->nA = counts[0];
  ctx->nV = counts[1];
  ctx->nR = counts[2];
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
  if (recapture) ctx->cg_graph_check = -1;
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
  return helm_solve(ctx, dt, stats);
}

int pyib_step(pyib_ctx* ctx, double dt, double dt_old, int32_t inner, const double* markers,
              const double* vel, pyib_step_stats* stats) {
  if (!ctx) return PYIB_E_ARG;
  if (!(dt > 0) || !(dt_old > 0)) return set_err(ctx, PYIB_E_ARG, "dt must be positive");
  if ((markers == nullptr) != (vel == nullptr)) return set_err(ctx, PYIB_E_ARG, "markers and vel go together");
  CK(cudaSetDevice(ctx->device));
  return do_step(ctx, dt, dt_old, inner, markers, vel, stats);
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
  double* dout = ctx->partials + (kSlots - 1) * kMaxBlocks;   // 13 doubles of scratch
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
  double* dout = ctx->partials + (kSlots - 1) * kMaxBlocks;
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
  if (reset) {
    ctx->cg_seconds = 0.0;
    ctx->cg_iters = 0;
    ctx->launches = 0;
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

int pyib_bench_matvec(pyib_ctx* ctx, int32_t reps, double dt, double* ms_per) {
  if (!ctx || reps <= 0 || !ms_per) return PYIB_E_ARG;
  if (!tables_ready(ctx) || !ctx->have_params) return set_err(ctx, PYIB_E_STATE, "context not ready");
  CK(cudaSetDevice(ctx->device));
  RET(set_state_solver(ctx, dt, 1));
  RET(launch_matvec(ctx, ctx->work_e, ctx->work_e2, 1, 0));   // warm
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  for (int q = 0; q < reps; ++q) RET(launch_matvec(ctx, ctx->work_e, ctx->work_e2, 1, 0));
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  *ms_per = ms / reps;
  return PYIB_OK;
}

}  // extern "C"
