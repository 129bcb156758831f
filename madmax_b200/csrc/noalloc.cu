// noalloc.cu -- sp_ell_pcg_noalloc: Jacobi-preconditioned CG on an ELL
// matrix that already lives in device memory, for callers that cannot
// allocate device memory.
//
// Who needs it: host frameworks that hand out all device memory from their
// own pool and forbid allocations behind their back, and latency-bound
// serving loops that must never enter the CUDA allocator (cudaMalloc and
// cudaFree synchronize the device and can stall for milliseconds).  Such a
// caller passes its matrix and vectors as device pointers it already owns;
// this entry point calls no cudaMalloc, cudaFree or other allocating
// routine.  Its work space (diagonal inverse, three CG vectors, reduction
// partials, scalars) is one file-scope __device__ array of fixed size, so at
// most SP_NOALLOC_MAX_ROWS rows fit.
//
// Set-up: the first call on a device, with that device current, looks up
// the array's device address with cudaGetSymbolAddress and keeps it; later
// calls check that the kept address is still a device address of that
// device (after a cudaDeviceReset it is not) and look it up again if not.
// Make the first call on a device before any stream capture begins.
//
// The array is shared by every call on a device and keeps the contents of
// the last call; each call clears what must start at zero.  Two calls whose
// GPU work overlaps (different streams, or different host threads) race on
// it: serialize them.
#include <cmath>
#include <mutex>

#include "sputnik_b200.h"
#include "sp_cuda.h"

namespace sp {
namespace noalloc {

constexpr int THREADS = 256;
constexpr int MAX_BLOCKS = 1024;

struct State {
  double rho, alpha, beta, bb, rr;
  double rtol2;
  int its, max_its, active;
  int bad;    // a column index outside [0, nrow) other than -1
  int zdiag;  // a row whose diagonal is zero or absent
  unsigned ticket;
};
static_assert(sizeof(State) <= 32 * sizeof(double), "State fits its slot of the work space");

// layout of the scratch array (doubles)
constexpr size_t OFF_STATE = 0;                                // State (padded to 32 doubles)
constexpr size_t OFF_PART = 32;                                // [MAX_BLOCKS][3]
constexpr size_t OFF_DINV = OFF_PART + 3 * MAX_BLOCKS;         // [max rows]
constexpr size_t OFF_R = OFF_DINV + SP_NOALLOC_MAX_ROWS;
constexpr size_t OFF_P = OFF_R + SP_NOALLOC_MAX_ROWS;
constexpr size_t OFF_Q = OFF_P + SP_NOALLOC_MAX_ROWS;
constexpr size_t SCRATCH_DOUBLES = OFF_Q + SP_NOALLOC_MAX_ROWS;

// every GPU that loads the library holds this array until exit
static __device__ __align__(256) double g_scratch[SCRATCH_DOUBLES];

// (A x)_row for a row-major ELL of any width, one warp per row.  Column
// indices outside [0, n) other than -1 are skipped and flagged in *bad.
__device__ inline double warp_row(int row, int n, int nnz, const int *cols, const double *vals,
                                  const double *x, int lane, int *bad) {
  double s = 0.0;
  for (int j = lane; j < nnz; j += 32) {
    int c = cols[(size_t)row * nnz + j];
    if (c >= 0 && c < n)
      s = fma(vals[(size_t)row * nnz + j], x[c], s);
    else if (c < -1 || c >= n)
      *bad = 1;
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  return s;
}

// The diagonal entry of a row (the sum of its slots in column row; 0 when
// there is none), by the whole warp; slots of -1 are skipped wherever they
// are, as warp_row skips them.
__device__ inline double warp_diag(int row, int nnz, const int *cols, const double *vals,
                                   int lane) {
  double d = 0.0;
  for (int j = lane; j < nnz; j += 32)
    if (cols[(size_t)row * nnz + j] == row) d += vals[(size_t)row * nnz + j];
  for (int off = 16; off > 0; off >>= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
  return d;
}

// Last-arriving block folds the per-block partials (3 per block) in block
// order.  Returns true in exactly one thread (thread 0 of the last block),
// the only one that holds the totals; it also resets the ticket.
__device__ inline bool fold3(double a, double b, double c, double *part, unsigned *ticket,
                             double *out) {
  __shared__ double sv[3][THREADS / 32];
  __shared__ bool last;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, off);
    b += __shfl_xor_sync(0xffffffffu, b, off);
    c += __shfl_xor_sync(0xffffffffu, c, off);
  }
  if (lane == 0) {
    sv[0][warp] = a;
    sv[1][warp] = b;
    sv[2][warp] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int v = 0; v < 3; v++) {
      double tv = 0.0;
      for (int w = 0; w < THREADS / 32; w++) tv += sv[v][w];
      part[3 * blockIdx.x + v] = tv;
    }
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return false;
  __threadfence();
  for (int v = 0; v < 3; v++) {
    double tv = 0.0;
    for (unsigned k = 0; k < gridDim.x; k++) tv += __ldcg(part + 3 * k + v);
    out[v] = tv;
  }
  *ticket = 0;
  return true;
}

// dinv, r = b - A x, p = z = dinv r; totals rho = r.z, bb = b.b
__global__ void __launch_bounds__(THREADS)
    k_start(int n, int nnz, const int *cols, const double *vals, const double *b,
            const double *x, double *S) {
  State *st = reinterpret_cast<State *>(S + OFF_STATE);
  double *dinv = S + OFF_DINV, *r = S + OFF_R, *p = S + OFF_P;
  int lane = threadIdx.x & 31;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double rz = 0.0, bb = 0.0, rr = 0.0;
  for (int row = warp; row < n; row += nw) {
    double ax = warp_row(row, n, nnz, cols, vals, x, lane, &st->bad);
    double diag = warp_diag(row, nnz, cols, vals, lane);
    if (lane == 0) {
      if (!(diag != 0.0)) st->zdiag = 1;  // zero, absent or NaN: no Jacobi inverse
      double di = (diag != 0.0) ? 1.0 / diag : 0.0, rv = b[row] - ax, z = di * rv;
      dinv[row] = di;
      r[row] = rv;
      p[row] = z;
      rz += rv * z;
      bb += b[row] * b[row];
      rr += rv * rv;
    }
  }
  double tot[3];
  if (fold3(rz, bb, rr, S + OFF_PART, &st->ticket, tot)) {
    st->rho = tot[0];
    st->bb = tot[1];
    st->rr = tot[2];
    st->its = 0;
    st->active = tot[1] > 0.0 && st->max_its > 0 && tot[2] > st->rtol2 * tot[1] && !st->bad &&
                 !st->zdiag && isfinite(tot[0]) && isfinite(tot[1]) && isfinite(tot[2]);
  }
}

// q = A p, alpha = rho / p.q
__global__ void __launch_bounds__(THREADS)
    k_spmv(int n, int nnz, const int *cols, const double *vals, double *S) {
  State *st = reinterpret_cast<State *>(S + OFF_STATE);
  if (!st->active || st->bad) return;
  const double *p = S + OFF_P;
  double *q = S + OFF_Q;
  int lane = threadIdx.x & 31;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  double pq = 0.0;
  for (int row = warp; row < n; row += nw) {
    double v = warp_row(row, n, nnz, cols, vals, p, lane, &st->bad);
    if (lane == 0) {
      q[row] = v;
      pq += p[row] * v;
    }
  }
  double tot[3];
  if (fold3(pq, 0.0, 0.0, S + OFF_PART, &st->ticket, tot))
    st->alpha = (tot[0] != 0.0) ? st->rho / tot[0] : 0.0;
}

// x += alpha p, r -= alpha q; convergence on r.r <= rtol^2 b.b; beta
__global__ void __launch_bounds__(THREADS) k_update(int n, double *x, double *S) {
  State *st = reinterpret_cast<State *>(S + OFF_STATE);
  if (!st->active) return;
  const double al = st->alpha;
  const double *dinv = S + OFF_DINV, *p = S + OFF_P, *q = S + OFF_Q;
  double *r = S + OFF_R;
  double rz = 0.0, rr = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += al * p[i];
    double rv = r[i] - al * q[i];
    r[i] = rv;
    rz += rv * dinv[i] * rv;
    rr += rv * rv;
  }
  double tot[3];
  if (fold3(rz, rr, 0.0, S + OFF_PART, &st->ticket, tot)) {
    st->rr = tot[1];
    st->its++;
    // a NaN or infinite residual is a breakdown: stop (the host reports it)
    if (tot[1] <= st->rtol2 * st->bb || st->its >= st->max_its || st->bad || !isfinite(tot[0]) ||
        !isfinite(tot[1])) {
      st->active = 0;
      st->beta = 0.0;
    } else {
      st->beta = (st->rho != 0.0) ? tot[0] / st->rho : 0.0;
      st->rho = tot[0];
    }
  }
}

// p = dinv r + beta p
__global__ void __launch_bounds__(THREADS) k_dir(int n, double *S) {
  State *st = reinterpret_cast<State *>(S + OFF_STATE);
  if (!st->active) return;
  const double be = st->beta;
  const double *dinv = S + OFF_DINV, *r = S + OFF_R;
  double *p = S + OFF_P;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = dinv[i] * r[i] + be * p[i];
}

static std::mutex g_mu;
static double *g_addr[64];

// whether p is still a device address of device dev (after a
// cudaDeviceReset the kept address belongs to a destroyed context)
static bool still_device_address(const double *p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

// the work space's device address, looked up once per device with that
// device current, and again when the kept one is no longer valid
static int scratch_address(int dev, double **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev] || !still_device_address(g_addr[dev], dev)) {
    double *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_scratch);
    if (e != cudaSuccess)
      return sp_set_error(SP_ERR_CUDA, "sp_ell_pcg_noalloc: cudaGetSymbolAddress failed: %s",
                          cudaGetErrorString(e));
    g_addr[dev] = ptr;
  }
  *out = g_addr[dev];
  return SP_OK;
}

}  // namespace noalloc
}  // namespace sp

using namespace sp;

extern "C" int sp_ell_pcg_noalloc(int nrow, int nnz, const int *cols_dev, const double *vals_dev,
                                  const double *b_dev, double *x_dev, double rtol, int max_its,
                                  int *its, double *relres, void *stream) {
  if (nrow < 1 || nnz < 1 || !cols_dev || !vals_dev || !b_dev || !x_dev || !(rtol > 0) ||
      max_its < 0)
    return sp_set_error(SP_ERR_ARG, "sp_ell_pcg_noalloc: bad argument");
  if (nrow > SP_NOALLOC_MAX_ROWS)
    return sp_set_error(SP_ERR_ARG,
                        "sp_ell_pcg_noalloc: %d rows exceed the fixed work space of %d rows", nrow,
                        SP_NOALLOC_MAX_ROWS);
  // the caller's current device; no library stream or other object is made
  int dev = -1, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return sp_set_error(SP_ERR_CUDA, "sp_ell_pcg_noalloc: no usable CUDA device");
  }
  double *S;
  SP_TRY(noalloc::scratch_address(dev, &S));
  cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : cudaStreamPerThread;
  noalloc::State st0 = {};
  st0.rtol2 = rtol * rtol;
  st0.max_its = max_its;
  // the scalars, including the reduction ticket, must start at zero
  SP_CUDA_TRY(cudaMemcpyAsync(S + noalloc::OFF_STATE, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
  int blocks = (nrow + 7) / 8;
  if (blocks > noalloc::MAX_BLOCKS) blocks = noalloc::MAX_BLOCKS;
  if (blocks > nsm * 4) blocks = nsm * 4;
  noalloc::k_start<<<blocks, noalloc::THREADS, 0, s>>>(nrow, nnz, cols_dev, vals_dev, b_dev, x_dev, S);
  SP_CUDA_TRY(cudaGetLastError());
  noalloc::State st;
  SP_CUDA_TRY(cudaMemcpyAsync(&st, S + noalloc::OFF_STATE, sizeof(st), cudaMemcpyDeviceToHost, s));
  SP_CUDA_TRY(cudaStreamSynchronize(s));
  // eight iterations per check; kernels of a finished solve return at once
  while (st.active) {
    for (int k = 0; k < 8; k++) {
      noalloc::k_spmv<<<blocks, noalloc::THREADS, 0, s>>>(nrow, nnz, cols_dev, vals_dev, S);
      noalloc::k_update<<<blocks, noalloc::THREADS, 0, s>>>(nrow, x_dev, S);
      noalloc::k_dir<<<blocks, noalloc::THREADS, 0, s>>>(nrow, S);
    }
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(cudaMemcpyAsync(&st, S + noalloc::OFF_STATE, sizeof(st), cudaMemcpyDeviceToHost, s));
    SP_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (its) *its = st.its;
  if (relres) *relres = (st.bb > 0) ? sqrt(st.rr / st.bb) : (st.bb == 0.0 ? 0.0 : NAN);
  if (st.bad)
    return sp_set_error(SP_ERR_RANGE, "sp_ell_pcg_noalloc: column index outside [0, nrow)");
  if (st.zdiag)
    return sp_set_error(SP_ERR_ARG, "sp_ell_pcg_noalloc: a row has a zero or no diagonal entry");
  // success only when the residual test holds (false for NaN): b = 0 is
  // solved by x = 0 only if the start iterate is 0
  const bool conv = (st.bb == 0.0) ? (st.rr == 0.0) : (st.rr <= st.rtol2 * st.bb);
  if (!conv)
    return sp_set_error(SP_ERR_NOCONV, "sp_ell_pcg_noalloc: no convergence in %d its (residual %g)",
                        st.its, st.bb > 0 ? sqrt(st.rr / st.bb) : sqrt(st.rr));
  return SP_OK;
}
