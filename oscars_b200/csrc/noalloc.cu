// noalloc.cu -- fixed-level FP64 flux that allocates no memory.
//
// Some callers cannot allocate device memory on the call path: a plugin that runs inside a host
// application's CUDA context where the application owns every allocation, or a real-time
// acquisition loop whose latency budget forbids a trip through the allocator after start-up.  For
// them this file offers one entry point whose scratch memory is a file-scope static __device__
// array, reserved when the library's module is loaded on a device and held until the process exits.
//
// The array's name is not a device address in host code.  Its address is looked up with
// cudaGetSymbolAddress, with the device current, once per device and CUDA context: the lookup is
// cached together with the context's unique ID, so a context that was destroyed and created again
// (cudaDeviceReset in the host application) gets a fresh lookup instead of a stale address.  The
// first call on a device (and the first after its context was re-created) does that lookup, so make
// it before any stream capture begins.  All calls share the one array and it keeps the previous
// call's contents: every region that must start at zero is cleared on each call, and two calls
// whose GPU work overlaps (from different host threads, or on a device another thread is also using
// through this entry point) race on the array.  Calls are synchronous: results are in `out` when the
// call returns, and the caller's current device is restored before every return.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <cuda_runtime.h>

#include "../../include/oscars_b200.h"
#include "host_core.h"
#include "kernels.h"

namespace {

constexpr size_t kScratchBytes = (size_t)16 << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;

// Address of g_noalloc_scratch per device, valid for the context whose unique ID it records.
struct ScratchSlot {
  unsigned long long ctx_id = 0;  // 0: not looked up
  void* addr = nullptr;
};
ScratchSlot g_slots[kMaxDevices];
std::mutex g_slots_mutex;

// Driver entry points for the current context's unique ID (cuCtxGetCurrent, cuCtxGetId, CUDA 12.0),
// resolved through the runtime so the library does not link libcuda directly.
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::once_flag g_driver_once;

// Unique ID of the current context, 0 if the driver cannot tell (the address is then looked up on
// every call).
unsigned long long current_context_id() {
  std::call_once(g_driver_once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!g_ctx_get_current || !g_ctx_get_id || g_ctx_get_current(&ctx) != 0 || !ctx || g_ctx_get_id(ctx, &id) != 0)
    return 0;
  return id;
}

// Device address of the scratch array on the current device (`device`), from the cache when the
// context is the one it was looked up in.
cudaError_t scratch_address(int device, void** out) {
  const unsigned long long id = current_context_id();
  std::lock_guard<std::mutex> lock(g_slots_mutex);
  ScratchSlot& slot = g_slots[device];
  if (id != 0 && slot.ctx_id == id && slot.addr) {
    *out = slot.addr;
    return cudaSuccess;
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  slot.ctx_id = id;
  slot.addr = p;
  *out = p;
  return cudaSuccess;
}

// Puts the caller's current device back when the entry point returns.
struct DeviceRestore {
  int prev = -1;
  ~DeviceRestore() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

void set_message(char* msg, long long cap, const char* text) {
  if (msg && cap > 0) std::snprintf(msg, (size_t)cap, "%s", text);
}

// Clamped cubic spline second derivatives of the 9 trajectory components, one thread per component,
// with the reference's operation order (include/TOMATH.h:141-203), rounding every step separately so
// the result equals the host spline bit for bit.  knots = [t | y(9) | y''(9)], u = 9 x n scratch.
__global__ void k_spline_second_derivatives(double* __restrict__ knots, double* __restrict__ u_all, int64_t n) {
  const int c = threadIdx.x;
  if (c >= 9) return;
  const double* X = knots;
  const double* Y = knots + (1 + c) * n;
  double* ypp = knots + (10 + c) * n;
  double* u = u_all + c * n;
  const double h0 = __dsub_rn(X[1], X[0]);
  const double dydx0 = __ddiv_rn(__dsub_rn(Y[1], Y[0]), h0);
  ypp[0] = -0.5;
  u[0] = __dmul_rn(__ddiv_rn(3., h0), __dsub_rn(__ddiv_rn(__dsub_rn(Y[1], Y[0]), h0), dydx0));
  for (int64_t i = 1; i < n - 1; ++i) {
    const double sig = __ddiv_rn(__dsub_rn(X[i], X[i - 1]), __dsub_rn(X[i + 1], X[i - 1]));
    const double p = __dadd_rn(__dmul_rn(sig, ypp[i - 1]), 2.0);
    ypp[i] = __ddiv_rn(__dsub_rn(sig, 1.), p);
    const double ui = __dsub_rn(__ddiv_rn(__dsub_rn(Y[i + 1], Y[i]), __dsub_rn(X[i + 1], X[i])),
                                __ddiv_rn(__dsub_rn(Y[i], Y[i - 1]), __dsub_rn(X[i], X[i - 1])));
    u[i] = __ddiv_rn(__dsub_rn(__ddiv_rn(__dmul_rn(6., ui), __dsub_rn(X[i + 1], X[i - 1])), __dmul_rn(sig, u[i - 1])), p);
  }
  const double hn = __dsub_rn(X[n - 1], X[n - 2]);
  const double dydxn = __ddiv_rn(__dsub_rn(Y[n - 1], Y[n - 2]), hn);
  const double un = __dmul_rn(__ddiv_rn(3., hn), __dsub_rn(dydxn, __ddiv_rn(__dsub_rn(Y[n - 1], Y[n - 2]), hn)));
  ypp[n - 1] = __ddiv_rn(__dsub_rn(un, __dmul_rn(0.5, u[n - 2])), __dadd_rn(__dmul_rn(0.5, ypp[n - 2]), 1.));
  for (int64_t j = n - 2; j >= 0; --j) ypp[j] = __dadd_rn(__dmul_rn(ypp[j], ypp[j + 1]), u[j]);
}

__global__ void k_store_double(double* p, double v) { *p = v; }

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" OSC_API int osc_flux_fixed_level_noalloc(int device, const double* trajectory, long long n_points,
                                                    const double* obs_xyz, long long n_obs, double energy_eV,
                                                    int level, double charge, double current,
                                                    const double polarization[6], double* out, char* message,
                                                    long long message_capacity) {
  using namespace osc;
  if (!trajectory || !obs_xyz || !out || n_points < 3 || n_obs < 1 || level < 0 || level > 30) {
    set_message(message, message_capacity, "invalid argument: need >= 3 trajectory points, >= 1 observer, level 0..30");
    return OSC_ERR_INVALID;
  }
  if (device < 0 || device >= kMaxDevices) {
    set_message(message, message_capacity, "device index out of range");
    return OSC_ERR_RANGE;
  }
  // scratch layout: knots (19 n) | spline work (9 n) | level samples (10 x 2^(level+1)) | observers
  // (3 n_obs) | omega | counters | per-level beta differences | results (n_obs) | span partials
  // (2 x 9 n_obs)
  const int64_t n = n_points;
  const int64_t cap = (int64_t)2 << level;
  const size_t off_knots = 0;
  const size_t off_u = align256(off_knots + sizeof(double) * 19 * n);
  const size_t off_lev = align256(off_u + sizeof(double) * 9 * n);
  const size_t off_obs = align256(off_lev + sizeof(double) * 10 * cap);
  const size_t off_omega = align256(off_obs + sizeof(double) * 3 * n_obs);
  const size_t off_cnt = align256(off_omega + sizeof(double));
  const size_t off_bd = align256(off_cnt + 8 * sizeof(unsigned long long));
  const size_t off_res = align256(off_bd + 32 * sizeof(unsigned long long));
  const size_t off_part = align256(off_res + sizeof(double) * n_obs);
  const WavePlan plan = wave_plan(1, level, n_obs, 128, 1, 32);  // one span: partials 2 x 9 per observer
  const size_t need = off_part + sizeof(double) * (size_t)plan.nseg * plan.spans * kFdPartials * n_obs;
  if (need > kScratchBytes) {
    char text[256];
    std::snprintf(text, sizeof text,
                  "request needs %zu bytes of scratch, above the 16 MiB static scratch of this entry point "
                  "(224 B per trajectory point + 80 B x 2^(level+1) + 176 B per observer)", need);
    set_message(message, message_capacity, text);
    return OSC_ERR_LENGTH;
  }
  DeviceRestore restore;
  cudaError_t e = cudaGetDevice(&restore.prev);
  if (e != cudaSuccess) restore.prev = -1;
  e = cudaSetDevice(device);
  void* scratch = nullptr;
  if (e == cudaSuccess) e = scratch_address(device, &scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_message(message, message_capacity, cudaGetErrorString(e));
    return OSC_ERR_CUDA;
  }
  unsigned char* base = static_cast<unsigned char*>(scratch);
  double* knots = reinterpret_cast<double*>(base + off_knots);
  double* u = reinterpret_cast<double*>(base + off_u);
  double* lev = reinterpret_cast<double*>(base + off_lev);
  double* obs = reinterpret_cast<double*>(base + off_obs);
  double* omega = reinterpret_cast<double*>(base + off_omega);
  unsigned* cnt = reinterpret_cast<unsigned*>(base + off_cnt);
  unsigned long long* c64 = reinterpret_cast<unsigned long long*>(base + off_cnt) + 2;
  unsigned long long* bd = reinterpret_cast<unsigned long long*>(base + off_bd);
  double* res = reinterpret_cast<double*>(base + off_res);
  double* part = reinterpret_cast<double*>(base + off_part);
  const cudaStream_t st = 0;  // legacy default stream; the call synchronises before returning

  const double tstart = trajectory[0], tstop = trajectory[n - 1];
  const double w = ev_to_omega(energy_eV);
  double pol[6] = {0, 0, 0, 0, 0, 0};
  if (polarization)
    for (int i = 0; i < 6; ++i) pol[i] = polarization[i];
  const double pm2 = (pol[0] * pol[0] + pol[1] * pol[1]) + (pol[2] * pol[2] + pol[3] * pol[3]) + (pol[4] * pol[4] + pol[5] * pol[5]);
  const double c0 = charge / (four_pi() * kC * kEps0 * kSqrt2Pi);                        // src/OSCARSSR.cc:4106
  const double c2 = four_pi() * current / (kH * std::fabs(charge) * kMu0 * kC) * 1e-6 * 0.001;  // :4109
  auto dt_inc = [&](int L) { return (tstop - tstart) / (std::pow(2., L + 1) - 1); };

  e = cudaMemcpyAsync(knots, trajectory, sizeof(double) * 10 * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(obs, obs_xyz, sizeof(double) * 3 * n_obs, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, 8 * sizeof(unsigned long long), st);  // counters and error word
  if (e == cudaSuccess) e = cudaMemsetAsync(bd, 0, 32 * sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    k_store_double<<<1, 1, 0, st>>>(omega, w);
    k_spline_second_derivatives<<<1, 32, 0, st>>>(knots, u, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = launch_level_fill(knots, n, tstart, tstop, 1, cap, lev, cap, kMaxLevelMemory, bd, st);
  if (e == cudaSuccess) {
    FdWaveArgs a{};
    a.lev = lev; a.cap = cap; a.obs = obs; a.omega = omega; a.n_e = 1; a.n_items = n_obs;
    a.act = nullptr; a.n_act = nullptr; a.first = 1; a.level = level; a.tile_entries = 128; a.min_span = 32;
    a.target_units = 1; a.part = part; a.err = cnt + 2; a.work = c64 + 2;  // zeroed with the counters
    e = launch_fd_wave_fp64(a, (int)(plan.tiles * plan.spans), 0, st);
  }
  if (e == cudaSuccess) {
    FdFinalArgs f{};
    f.part = part; f.first = 1; f.level = level; f.max_level = level; f.quantity = 0;
    f.project = pm2 > 0.001; f.tile_entries = 128; f.min_span = 32; f.target_units = 1;
    f.dt_prev = level >= 1 ? dt_inc(level - 1) : 0; f.dt_level = dt_inc(level);
    f.precision = 0; f.c0 = c0; f.c2 = c2; f.weight = 1;
    for (int i = 0; i < 6; ++i) f.pol[i] = pol[i];
    f.n_items = n_obs; f.act = nullptr; f.n_act = nullptr; f.state = u;  // never written at the last level
    f.act_next = reinterpret_cast<int*>(u); f.n_next = cnt + 1;
    f.out = res; f.level_out = nullptr; f.not_converged = c64; f.samples = c64 + 1; f.work_reset = c64 + 2;
    e = launch_fd_finalize(f, n_obs, st);
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, res, sizeof(double) * n_obs, cudaMemcpyDeviceToHost);
  unsigned err_word = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&err_word, cnt + 2, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_message(message, message_capacity, cudaGetErrorString(e));
    return OSC_ERR_CUDA;
  }
  if (err_word) {
    set_message(message, message_capacity, "a staged trajectory copy did not complete (device wait limit reached)");
    return OSC_ERR_TIMEOUT;
  }
  set_message(message, message_capacity, "");
  return OSC_OK;
}
