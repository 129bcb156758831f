// device.cu -- device selection, the library stream, and the cache of
// device-resident mesh plans (one per distinct RVE mesh size).
#include <mutex>
#include <vector>

#include "sp_cuda.h"

namespace sp {

static std::mutex g_mu;
static Device g_devs[64];
static thread_local int t_dev = 0;

int device(Device **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return sp_set_error(SP_ERR_CUDA, "no usable CUDA device (%s)",
                        e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
  }
  if (t_dev < 0 || t_dev >= n || t_dev >= 64)
    return sp_set_error(SP_ERR_CUDA, "device %d not present (%d devices)", t_dev, n);
  Device &d = g_devs[t_dev];
  SP_CUDA_TRY(cudaSetDevice(t_dev));
  if (d.id < 0) {
    cudaDeviceProp prop;
    SP_CUDA_TRY(cudaGetDeviceProperties(&prop, t_dev));
    if (prop.major < 10)
      return sp_set_error(SP_ERR_CUDA, "device %d is sm_%d%d; this build targets sm_100a", t_dev,
                          prop.major, prop.minor);
    d.nsm = prop.multiProcessorCount;
    SP_CUDA_TRY(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
    d.id = t_dev;
  }
  *out = &d;
  return SP_OK;
}

cudaStream_t pick_stream(void *user_stream, Device *d) {
  return user_stream ? reinterpret_cast<cudaStream_t>(user_stream) : d->stream;
}

int dmalloc(void **p, size_t bytes, size_t *acct) {
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return sp_set_error(SP_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  if (acct) *acct += bytes;
  return SP_OK;
}

MeshGeo make_geo(const int *n, const double *len) {
  MeshGeo g;
  g.nex = n[0];
  g.ney = n[1];
  g.nez = n[2];
  g.nx = n[0] + 1;
  g.ny = n[1] + 1;
  g.nz = n[2] + 1;
  g.nn = g.nx * g.ny * g.nz;
  g.nn_pad = (g.nn + 31) / 32 * 32;
  g.ndof = 3 * g.nn;
  g.nelm = n[0] * n[1] * n[2];
  g.hx = len[0] / n[0];
  g.hy = len[1] / n[1];
  g.hz = len[2] / n[2];
  g.vol = len[0] * len[1] * len[2];
  g.periodic = 0;
  g.pad = 0;
  return g;
}

size_t plan_bytes(const int *n) {
  size_t nn = (size_t)(n[0] + 1) * (n[1] + 1) * (n[2] + 1);
  size_t ndof = 3 * nn, nn_pad = (nn + 31) / 32 * 32;
  size_t nelm = (size_t)n[0] * n[1] * n[2];
  return ndof * SP_WP * sizeof(int) + nelm * SP_KE + nelm * sizeof(int) +
         nn_pad * 27 * sizeof(int);
}

static std::vector<DevPlan *> g_plans;

int plan_acquire(const int *n, DevPlan **out) {
  Device *d;
  SP_TRY(device(&d));
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (DevPlan *p : g_plans)
      if (p->dev == d->id && p->n[0] == n[0] && p->n[1] == n[1] && p->n[2] == n[2]) {
        p->refs++;
        *out = p;
        return SP_OK;
      }
  }
  sp_plan_host h;
  SP_TRY(sp_plan_build(n, &h));
  DevPlan *p = new DevPlan();
  for (int k = 0; k < 3; k++) p->n[k] = n[k];
  double one[3] = {1.0, 1.0, 1.0};
  p->geo = make_geo(n, one);
  for (int c = 0; c < 9; c++) p->color_off[c] = h.color_off[c];
  p->boundary_nodes = h.boundary_nodes;
  p->dev = d->id;
  size_t cb = (size_t)h.ndof * SP_WP * sizeof(int), sb = (size_t)h.nelm * SP_KE,
         eb = (size_t)h.nelm * sizeof(int), nb = (size_t)h.nslice * 27 * 32 * sizeof(int);
  int rc = dmalloc((void **)&p->cols, cb, &p->bytes);
  if (!rc) rc = dmalloc((void **)&p->slot, sb, &p->bytes);
  if (!rc) rc = dmalloc((void **)&p->color_elems, eb, &p->bytes);
  if (!rc) rc = dmalloc((void **)&p->nbr, nb, &p->bytes);
  if (!rc) {
    cudaError_t e1 = cudaMemcpy(p->cols, h.cols, cb, cudaMemcpyHostToDevice);
    cudaError_t e2 = cudaMemcpy(p->slot, h.slot, sb, cudaMemcpyHostToDevice);
    cudaError_t e3 = cudaMemcpy(p->color_elems, h.color_elems, eb, cudaMemcpyHostToDevice);
    cudaError_t e4 = cudaMemcpy(p->nbr, h.nbr, nb, cudaMemcpyHostToDevice);
    if (e1 || e2 || e3 || e4) rc = sp_set_error(SP_ERR_CUDA, "plan upload failed");
  }
  sp_plan_free(&h);
  if (rc) {
    cudaFree(p->nbr);
    cudaFree(p->cols);
    cudaFree(p->slot);
    cudaFree(p->color_elems);
    delete p;
    return rc;
  }
  p->refs = 1;
  std::lock_guard<std::mutex> lk(g_mu);
  g_plans.push_back(p);
  *out = p;
  return SP_OK;
}

void plan_release(DevPlan *p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if (--p->refs > 0) return;
  for (size_t i = 0; i < g_plans.size(); i++)
    if (g_plans[i] == p) {
      g_plans.erase(g_plans.begin() + i);
      break;
    }
  int cur = -1;
  cudaGetDevice(&cur);
  cudaSetDevice(p->dev);
  cudaFree(p->nbr);
  cudaFree(p->cols);
  cudaFree(p->slot);
  cudaFree(p->color_elems);
  if (cur >= 0) cudaSetDevice(cur);
  delete p;
}

}  // namespace sp

extern "C" int sp_init(int device) {
  if (device < 0) return sp_set_error(SP_ERR_ARG, "negative device id");
  sp::t_dev = device;
  sp::Device *d;
  return sp::device(&d);
}

extern "C" int sp_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}
