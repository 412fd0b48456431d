// Batched conserved-to-primitive inversion that allocates nothing.
//
// kgpu_u2p_cells() stages its inputs in device buffers obtained from
// cudaMalloc for every call.  Some hosts cannot do that at the point where
// they invert cells: a caller whose device memory is owned by another
// allocator or pool, one running inside a region where an allocation's
// implicit device-wide synchronisation would stall other streams, or a
// long-running service that must not grow or fragment the device heap.
// kgpu_u2p_cells_static() serves them: its staging area is a file-scope
// device array of fixed size, so neither the call nor its first-call set-up
// allocates host or device memory.
//
// Limits and behaviour
//  - At most KGPU_STATIC_MAX_CELLS cells per call; larger batches are
//    rejected with KGPU_EINVAL and an error message (split them).
//  - The array lives in every GPU that loads this library until the process
//    exits (KGPU_STATIC_MAX_CELLS * 472 bytes, about 3.9 MB).
//  - The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (that device current); make that first call before
//    any stream capture.  The address is kept per device together with the
//    identity of the device's CUDA context: after cudaDeviceReset (or any
//    other teardown and re-creation of the context, which reloads the module
//    and moves the array) the next call looks the address up again, so
//    that call, too, belongs before any stream capture.
//  - All calls share the one array, which keeps the last call's contents.
//    Every word the kernel reads is written by the same call's copies, so no
//    clearing is needed; calls that overlap on the GPU (from several host
//    threads) race on the array and must be serialised by the caller.
//  - Copies are synchronous on the legacy default stream.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "../../include/koral_b200.h"
#include "kgpu_physics.cuh"

using namespace kgpu;

namespace {

constexpr int kNV = 9;
static_assert(NVMAX == kNV, "the static batch carries the nine MHD variables");
constexpr int kCellBytes = (9 + 9 + 20 + 20) * 8 + 2 * 4;   // uu, pp, g, G, status, fixup
constexpr size_t kScratchBytes = (size_t)KGPU_STATIC_MAX_CELLS * kCellBytes;

// region offsets inside the array for n cells (each region 256-byte aligned)
inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
struct Layout {
  size_t uu, pp, g, G, st, fx, end;
  explicit Layout(int n) {
    uu = 0;
    pp = align256(uu + (size_t)n * 9 * 8);
    g = align256(pp + (size_t)n * 9 * 8);
    G = align256(g + (size_t)n * 20 * 8);
    st = align256(G + (size_t)n * 20 * 8);
    fx = align256(st + (size_t)n * 4);
    end = align256(fx + (size_t)n * 4);
  }
};

}  // namespace

// The staging array.  Host code never takes its address directly (that would
// be the host shadow); the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char kgpu_static_scratch[kScratchBytes + 6 * 256];

namespace {

constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices];            // device address per device ordinal ...
unsigned long long g_scratch_ctx[kMaxDevices];  // ... and the context it was looked up in
std::mutex g_setup_mutex;
thread_local char g_err[200];

// Unique identity of the current context (cuCtxGetId: unique over the
// process's lifetime, unlike the context handle, which a re-created context
// may reuse), through the runtime's driver entry points so that the
// library needs no link to the driver library.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext *);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long *);
int current_context_id(unsigned long long *id) {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  if (!get_current || !get_id) {
    cudaDriverEntryPointQueryResult q1, q2;
    void *f1 = nullptr, *f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || !f1 ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess || !f2) {
      snprintf(g_err, sizeof(g_err), "driver entry points cuCtxGetCurrent/cuCtxGetId not found");
      return KGPU_ECUDA;
    }
    get_current = (PfnCtxGetCurrent)f1;
    get_id = (PfnCtxGetId)f2;
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS) {
    snprintf(g_err, sizeof(g_err), "no current CUDA context");
    return KGPU_ECUDA;
  }
  return 0;
}

int scratch_for_current_device(unsigned char **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    snprintf(g_err, sizeof(g_err), "cudaGetDevice: %s", cudaGetErrorString(e));
    return KGPU_ECUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    snprintf(g_err, sizeof(g_err), "device ordinal %d beyond %d", dev, kMaxDevices);
    return KGPU_EINVAL;
  }
  // makes the device's primary context current (and creates it on first use)
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) {
    snprintf(g_err, sizeof(g_err), "context set-up: %s", cudaGetErrorString(e));
    return KGPU_ECUDA;
  }
  unsigned long long ctx = 0;
  int r = current_context_id(&ctx);
  if (r) return r;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, kgpu_static_scratch);
    if (e != cudaSuccess || !p) {
      snprintf(g_err, sizeof(g_err), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return KGPU_ECUDA;
    }
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = (unsigned char *)g_scratch_addr[dev];
  return 0;
}

}  // namespace

// same inversion as k_u2p_cells, reading KORAL's cell-major layout directly
__global__ void k_u2p_cells_aos(Grid G, int n, const double *uu, double *pp, const double *g20, const double *G20,
                                int *status, int *fixup) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Geom g;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 5; b++) {
      g.gg[a][b] = g20[(long)i * 20 + a * 5 + b];
      g.GG[a][b] = G20[(long)i * 20 + a * 5 + b];
    }
  g.gdet = g.gg[3][4];
  g.gttpert = g.GG[3][4];
  double u[kNV], p[kNV];
  for (int iv = 0; iv < kNV; iv++) {
    u[iv] = uu[(long)i * kNV + iv];
    p[iv] = pp[(long)i * kNV + iv];
  }
  int fix = 0;
  int ret = u2p(G, u, p, g, fix);
  for (int iv = 0; iv < kNV; iv++) pp[(long)i * kNV + iv] = p[iv];
  status[i] = ret;
  fixup[i] = fix;
}

extern "C" const char *kgpu_u2p_cells_static_error(void) { return g_err; }

extern "C" int kgpu_u2p_cells_static(int n, const kgpu_config *cfg, const double *uu, double *pp, const double *g,
                                     const double *Gi, int *status, int *fixup) {
  g_err[0] = 0;
  if (n < 0 || !cfg || (n > 0 && (!uu || !pp || !g || !Gi || !status || !fixup)) || cfg->nv != 9) {
    snprintf(g_err, sizeof(g_err), "invalid argument");
    return KGPU_EINVAL;
  }
  if (n > KGPU_STATIC_MAX_CELLS) {
    snprintf(g_err, sizeof(g_err), "%d cells exceed the static limit of %d per call", n, KGPU_STATIC_MAX_CELLS);
    return KGPU_EINVAL;
  }
  if (n == 0) return 0;
  unsigned char *base = nullptr;
  int r = scratch_for_current_device(&base);
  if (r) return r;
  Grid G;
  memset(&G, 0, sizeof(G));
  G.nv = 9;
  G.gamma = cfg->gamma;
  G.rhofloor = cfg->rhofloor;
  G.uurhoratiomin = cfg->uurhoratiomin;
  G.uurhoratiomax = cfg->uurhoratiomax;
  G.b2rhoratiomax = cfg->b2rhoratiomax;
  G.gammamaxhd = cfg->gammamaxhd;
  G.u2pconv = cfg->u2pconv;
  Layout L(n);
  if (L.end > sizeof(kgpu_static_scratch)) {   // cannot happen for n <= KGPU_STATIC_MAX_CELLS
    snprintf(g_err, sizeof(g_err), "static layout of %d cells overruns the array", n);
    return KGPU_EINVAL;
  }
  double *duu = (double *)(base + L.uu), *dpp = (double *)(base + L.pp);
  double *dg = (double *)(base + L.g), *dG = (double *)(base + L.G);
  int *dst = (int *)(base + L.st), *dfx = (int *)(base + L.fx);
  cudaError_t e;
#define SCK(call)                                                                    \
  do {                                                                               \
    e = (call);                                                                      \
    if (e != cudaSuccess) {                                                          \
      snprintf(g_err, sizeof(g_err), "%s: %s", #call, cudaGetErrorString(e));        \
      return KGPU_ECUDA;                                                             \
    }                                                                                \
  } while (0)
  SCK(cudaMemcpy(duu, uu, (size_t)n * 9 * 8, cudaMemcpyHostToDevice));
  SCK(cudaMemcpy(dpp, pp, (size_t)n * 9 * 8, cudaMemcpyHostToDevice));
  SCK(cudaMemcpy(dg, g, (size_t)n * 20 * 8, cudaMemcpyHostToDevice));
  SCK(cudaMemcpy(dG, Gi, (size_t)n * 20 * 8, cudaMemcpyHostToDevice));
  k_u2p_cells_aos<<<(n + 127) / 128, 128>>>(G, n, duu, dpp, dg, dG, dst, dfx);
  SCK(cudaGetLastError());
  SCK(cudaMemcpy(pp, dpp, (size_t)n * 9 * 8, cudaMemcpyDeviceToHost));
  SCK(cudaMemcpy(status, dst, (size_t)n * 4, cudaMemcpyDeviceToHost));
  SCK(cudaMemcpy(fixup, dfx, (size_t)n * 4, cudaMemcpyDeviceToHost));
#undef SCK
  return 0;
}
