// engine.cu -- device state of one context and the wave scheduler of the radiation integrals.
//
// Data layout in HBM for one trajectory:
//   knots   19 x n doubles: t, y[9] (x y z, beta, a/c), y''[9]      (from the host RK4 + spline)
//   levels  10 x cap doubles, cap = 2^(Lmax+1): level L sample i at index 2^L + i
// Per request: observers (3 x n_obs), angular frequencies, per-entry state (running complex sum and
// last magnitude), two active-entry lists, span partials, outputs.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <exception>
#include <mutex>
#include <thread>

#include "kernels.h"

namespace osc {

namespace {
// Compensated accumulation of one particle's values (T3DScalarContainer::AddToPoint,
// src/T3DScalarContainer.cc:35-51), unfused like the reference.
__global__ void k_kahan_add(double* sum, double* comp, const double* v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double S = sum[i];
  const double y = __dsub_rn(v[i], comp[i]);
  const double t = __dadd_rn(S, y);
  comp[i] = __dsub_rn(__dsub_rn(t, S), y);
  sum[i] = t;
}
}  // namespace

void DevBuf::reserve(size_t n) {
  if (n <= bytes) return;
  release();
  if (cudaMalloc(&p, n) != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    cudaGetLastError();
    throw Error{OSC_ERR_ALLOC, "device allocation of " + std::to_string(n) + " bytes failed"};
  }
  bytes = n;
}
void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

Engine::Engine(int dev) : device(dev) {
  if (dev < 0) return;  // host-only context: model, trajectory and surfaces, no radiation calls
  check(cudaSetDevice(dev), "cudaSetDevice");
  check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  bd_bits_.reserve(32 * sizeof(unsigned long long));
  mrec_bd_.reserve(32 * sizeof(unsigned long long));
  cnt_.reserve(64);
  check(cudaMemset(cnt_.p, 0, 64), "memset");
  check(cudaHostAlloc(reinterpret_cast<void**>(&stats_host_), kStatWords * kStatSlots * sizeof(unsigned long long),
                      cudaHostAllocMapped),
        "cudaHostAlloc");
  check(cudaHostAlloc(reinterpret_cast<void**>(&stage_host_), kStageDoubles * sizeof(double), cudaHostAllocMapped),
        "cudaHostAlloc");
  check(cudaHostAlloc(reinterpret_cast<void**>(&ctl_host_), 16 * sizeof(unsigned), cudaHostAllocMapped),
        "cudaHostAlloc");
  for (int i = 0; i < kStatSlots; ++i) check(cudaEventCreateWithFlags(&stats_ev_[i], cudaEventDisableTiming), "event");
  check(cudaEventCreateWithFlags(&stage_ev_, cudaEventDisableTiming), "event");
  check(cudaEventCreateWithFlags(&order_ev_, cudaEventDisableTiming), "event");
  check(cudaStreamCreateWithFlags(&aux_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming), "event");
  check(cudaEventCreateWithFlags(&join_ev_, cudaEventDisableTiming), "event");
  check(cudaEventCreateWithFlags(&zs_fork_ev_, cudaEventDisableTiming), "event");
  check(cudaEventCreateWithFlags(&zs_ev_, cudaEventDisableTiming), "event");
  check(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking), "cudaStreamCreate");
  for (cudaEvent_t* e : {&in_fork_ev_, &in_ev_})
    check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "event");
  cur_ = stream;
}

Engine::~Engine() {
  if (device < 0) return;
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  if (aux_) cudaStreamSynchronize(aux_);
  if (copy_) cudaStreamSynchronize(copy_);
  for (auto& e : ev_pending_) { ev_pool_.push_back(e.first); ev_pool_.push_back(e.second); }
  for (cudaEvent_t e : ev_pool_) cudaEventDestroy(e);
  for (int i = 0; i < kStatSlots; ++i) if (stats_ev_[i]) cudaEventDestroy(stats_ev_[i]);
  if (stage_ev_) cudaEventDestroy(stage_ev_);
  if (order_ev_) cudaEventDestroy(order_ev_);
  if (fork_ev_) cudaEventDestroy(fork_ev_);
  if (join_ev_) cudaEventDestroy(join_ev_);
  if (zs_fork_ev_) cudaEventDestroy(zs_fork_ev_);
  if (zs_ev_) cudaEventDestroy(zs_ev_);
  for (cudaEvent_t e : {in_fork_ev_, in_ev_})
    if (e) cudaEventDestroy(e);
  if (last_stream_valid_ && last_stream_ != stream) cudaStreamSynchronize(last_stream_);
  if (stats_host_) cudaFreeHost(stats_host_);
  if (stage_host_) cudaFreeHost(stage_host_);
  if (ctl_host_) cudaFreeHost(ctl_host_);
  for (PinnedStage& p : pin_pool_) {
    if (p.copied) {
      cudaEventSynchronize(p.copied);
      cudaEventDestroy(p.copied);
    }
    if (p.pinned) cudaFreeHost(p.pinned);
  }
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  for (DevBuf* b : {&knots_, &lev_, &bd_bits_, &mrec_bd_, &obs_, &nrm_, &omega_, &out_, &lvl_, &state_, &part_, &act_[0],
                    &act_[1], &cnt_, &acc_, &acc_comp_, &mrec_, &b_fields_, &b_fvals_, &b_obs_, &b_omega_, &b_acc_, &b_jobs_,
                    &b_knots_, &b_work_, &b_rec_, &b_rec_ext_, &b_state_, &b_out_, &b_lvl_, &b_act_[0], &b_act_[1],
                    &b_part_, &b_plan_, &b_cnt_, &adj_, &adj_s_, &adj_r_, &adj_sums_, &adj_z_, &fused_, &stl_geo_,
                    &stl_cen_, &stl_nrm_,
                    &stl_state_, &stl_flags_})
    b->release();
  if (stream) cudaStreamDestroy(stream);
  if (aux_) cudaStreamDestroy(aux_);
  if (copy_) cudaStreamDestroy(copy_);
}

void Engine::check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error{OSC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

void Engine::upload_trajectory(const double* pinned) {
  const Knots& k = model.knots;
  if (knots_version_ == model.knots_version && nknots_ == k.n) return;
  levels_dropped_ = false;
  const int64_t n = k.n;
  join_rk4_states(cur_);  // the side stream may still read the knots
  knots_.reserve(sizeof(double) * 20 * n);
  double* d = knots_.as<double>();
  if (pinned) {  // the same knots already laid out in pinned memory: one asynchronous copy
    check(cudaMemcpyAsync(d, pinned, sizeof(double) * 20 * n, cudaMemcpyHostToDevice, cur_), "upload knots");
  } else {
    check(cudaMemcpyAsync(d, k.t.data(), sizeof(double) * n, cudaMemcpyHostToDevice, cur_), "upload t");
    check(cudaMemcpyAsync(d + n, k.y.data(), sizeof(double) * 9 * n, cudaMemcpyHostToDevice, cur_), "upload y");
    check(cudaMemcpyAsync(d + 10 * n, k.ypp.data(), sizeof(double) * 9 * n, cudaMemcpyHostToDevice, cur_),
          "upload ypp");
    if ((int64_t)k.diag.size() == n)
      check(cudaMemcpyAsync(d + 19 * n, k.diag.data(), sizeof(double) * n, cudaMemcpyHostToDevice, cur_),
            "upload diag");
  }
  nknots_ = n;
  tstart_ = k.tstart;
  tstop_ = k.tstop;
  knots_version_ = model.knots_version;
  lev_filled_ = -1;
  mrec_filled_ = -1;
  bdmax_valid_ = false;
  check(cudaMemsetAsync(bd_bits_.p, 0, 32 * sizeof(unsigned long long), cur_), "memset");
}

// Capacity of the FP64 level cache for levels 0..L; growing keeps what is filled (the 10 arrays are
// copied into the larger cache).
void Engine::reserve_levels(int L) {
  const int64_t need = (int64_t)2 << L;
  if (need <= lev_cap_) return;
  int64_t cap = std::max<int64_t>(need, (int64_t)2 << 13);
  if (lev_cap_ > 0 && lev_filled_ >= 0) {
    DevBuf nb;
    nb.reserve(sizeof(double) * 10 * cap);
    const int64_t used = (int64_t)2 << lev_filled_;
    for (int a = 0; a < 10; ++a)
      check(cudaMemcpyAsync(nb.as<double>() + a * cap, lev_.as<double>() + a * lev_cap_, sizeof(double) * used,
                            cudaMemcpyDeviceToDevice, cur_),
            "level cache grow");
    check(cudaStreamSynchronize(cur_), "level cache grow");
    lev_.release();
    lev_ = nb;
    nb.p = nullptr;
  } else {
    lev_.reserve(sizeof(double) * 10 * cap);
  }
  lev_cap_ = cap;
}

void Engine::fill_levels(int64_t s_begin, int64_t s_end, cudaStream_t s) {
  check(launch_level_fill(knots_.as<double>(), nknots_, tstart_, tstop_, s_begin, s_end, lev_.as<double>(), lev_cap_,
                          lev_ext_, bd_bits_.as<unsigned long long>(), s),
        "level fill");
  ++last_launches;
  bdmax_valid_ = false;
}

// Levels above ext_from are the reference's extended levels (src/OSCARSSR.cc:4181-4186: above
// LevelStopMemory = max_level the levels are evaluated on the fly with their own time spacing,
// level_time in fd_common.cuh).  Cached levels whose times differ under the new split are dropped.
void Engine::set_level_grid(int ext_from) {
  if (ext_from != lev_ext_) {
    const int keep = std::min(ext_from, lev_ext_);
    if (lev_filled_ > keep) {
      lev_filled_ = keep;
      bdmax_valid_ = false;
      // the beta-difference maxima of the dropped levels are folded again by their refill
      check(cudaMemsetAsync(bd_bits_.as<unsigned long long>() + keep + 1, 0, sizeof(unsigned long long) * (31 - keep),
                            cur_),
            "memset");
      ++last_launches;
    }
    lev_ext_ = ext_from;
  }
  if (ext_from != mrec_ext_) {
    mrec_filled_ = std::min(mrec_filled_, std::min(ext_from, mrec_ext_));
    mrec_ext_ = ext_from;
  }
}

// Last level of a request and the split between the reference's memory levels and its extended
// levels (src/OSCARSSR.cc:4108-4109): LevelStopMemory = max_level (within [-1, 26]), levels up to
// max(max_level_extended, LevelStopMemory).  Returns the last level; `ext_from` is the highest level
// on the memory grid (26 when no extended level is used, so requests without them share the cache).
int request_levels(const osc_rad_opts& o, int max_supported, int* ext_from) {
  const int lstop_mem = o.max_level >= -1 && o.max_level <= kMaxLevelMemory ? o.max_level : kMaxLevelMemory;
  const int lstop = o.max_level_extended > lstop_mem ? o.max_level_extended : lstop_mem;
  if (lstop > max_supported)
    throw Error{OSC_ERR_RANGE, "max_level_extended above " + std::to_string(max_supported) +
                                   " is not supported by this GPU build for this calculation"};
  if (lstop < 0) throw Error{OSC_ERR_RANGE, "max_level -1 selects only extended levels, which this GPU build does not support"};
  *ext_from = lstop > lstop_mem ? lstop_mem : kMaxLevelMemory;
  return lstop;
}

// Make levels 0..L resident.
void Engine::ensure_levels(int L) {
  if (L <= lev_filled_) return;
  reserve_levels(L);
  if (lev_filled_ < 0) {
    check(cudaMemsetAsync(bd_bits_.p, 0, 32 * sizeof(unsigned long long), cur_), "memset");
    ++last_launches;
  }
  fill_levels(lev_filled_ < 0 ? 1 : ((int64_t)2 << lev_filled_), (int64_t)2 << L, cur_);
  lev_filled_ = L;
}

// Frame of the mixed path (kernels_mixed.cu): origin at the particle start, e3 along its initial
// velocity, e1 = unit(Orthogonal(e3)), e2 = e3 x e1; trajectory extent measured on the knots.
void Engine::compute_frame() {
  const Particle& P = model.particle;
  const Vec3 e3 = unit(P.b0);
  const Vec3 e1 = unit(orthogonal(e3));
  const Vec3 e2 = cross(e3, e1);
  const Vec3 rows[3] = {e1, e2, e3};
  for (int r = 0; r < 3; ++r) {
    frame_.rot[3 * r] = rows[r].x;
    frame_.rot[3 * r + 1] = rows[r].y;
    frame_.rot[3 * r + 2] = rows[r].z;
  }
  frame_.x0[0] = P.x0.x; frame_.x0[1] = P.x0.y; frame_.x0[2] = P.x0.z;
  frame_.t_ref = P.t0 / kC;
  const Knots& k = model.knots;
  double xp = 0, zm = -1e300, tm = 0;
  for (int64_t i = 0; i < k.n; ++i) {
    const Vec3 d = v3(k.y[i] - P.x0.x, k.y[k.n + i] - P.x0.y, k.y[2 * k.n + i] - P.x0.z);
    const double a = dot(d, e1), b = dot(d, e2), c = dot(d, e3);
    xp = std::max(xp, std::sqrt(a * a + b * b));
    zm = std::max(zm, c);
    tm = std::max(tm, std::fabs((k.t[i] - frame_.t_ref) - c / kC));
  }
  frame_.xperp_max = xp;
  frame_.z_max = zm;
  frame_.tau_max = tm;
  frame_.theta_max = mixed_theta_max(P.gamma);
}

// Capacity of the mixed pair records for levels 0..L (the frame is set up for the current knots
// first); growing refills from sample 0 (one spline evaluation per sample).
void Engine::reserve_mixed(int L) {
  if (mrec_version_ != knots_version_) {
    compute_frame();
    mrec_version_ = knots_version_;
    mrec_filled_ = -1;
  }
  const int64_t need = (int64_t)2 << L;
  if (need <= mrec_cap_) return;
  const int64_t cap = std::max<int64_t>(need, (int64_t)2 << 14);
  mrec_.release();
  mrec_.reserve((size_t)kMixedRecordBytesPerSample * cap);
  mrec_cap_ = cap;
  mrec_filled_ = -1;
}

void Engine::fill_mixed(int64_t s_begin, int64_t s_end, cudaStream_t s, bool zero_bd) {
  if (s_end <= s_begin) return;
  // the beta-difference maxima of the levels filled here start from zero
  if (zero_bd) {
    const int Lb = s_begin <= 1 ? 0 : 63 - __builtin_clzll((unsigned long long)s_begin);
    const int Le = 63 - __builtin_clzll((unsigned long long)(s_end - 1));
    check(cudaMemsetAsync(mrec_bd_.as<unsigned long long>() + Lb, 0, sizeof(unsigned long long) * (Le - Lb + 1), s),
          "memset");
    ++last_launches;
  }
  check(launch_mixed_records(knots_.as<double>(), nknots_, tstart_, tstop_, s_begin, s_end, mrec_ext_, frame_,
                             mrec_.as<float4>(), mrec_bd_.as<unsigned long long>(), s),
        "mixed records");
  ++last_launches;
}

void Engine::ensure_mixed(int L) {
  reserve_mixed(L);
  if (L <= mrec_filled_) return;
  fill_mixed(mrec_filled_ < 0 ? 0 : ((int64_t)2 << mrec_filled_), (int64_t)2 << L, cur_);
  mrec_filled_ = L;
}

// Levels 0..Lpre resident for the waves enqueued without a host round trip.  The levels above the
// first wave's (Lhead) are filled on the side stream, concurrently with the first wave; join_prefill()
// makes the request stream wait for them before the second wave.
void Engine::prefill(bool mixed, int Lhead, int Lpre, bool bd_zeroed) {
  if (mixed) reserve_mixed(Lpre);
  else reserve_levels(Lpre);
  int& filled = mixed ? mrec_filled_ : lev_filled_;
  if (Lpre <= filled) return;
  if (!mixed && filled < 0 && !bd_zeroed) {
    check(cudaMemsetAsync(bd_bits_.p, 0, 32 * sizeof(unsigned long long), cur_), "memset");
    ++last_launches;
  }
  const int lo = std::max(filled, Lhead);
  if (Lpre > lo) {
    check(cudaEventRecord(fork_ev_, cur_), "event");
    check(cudaStreamWaitEvent(aux_, fork_ev_, 0), "stream wait");
    if (mixed) fill_mixed((int64_t)2 << lo, (int64_t)2 << Lpre, aux_, !bd_zeroed);
    else fill_levels((int64_t)2 << lo, (int64_t)2 << Lpre, aux_);
    check(cudaEventRecord(join_ev_, aux_), "event");
    join_pending_ = true;
  }
  if (lo > filled) {
    const int64_t b = filled < 0 ? (mixed ? 0 : 1) : ((int64_t)2 << filled);
    if (mixed) fill_mixed(b, (int64_t)2 << lo, cur_, !bd_zeroed);
    else fill_levels(b, (int64_t)2 << lo, cur_);
  }
  filled = Lpre;
}

void Engine::join_prefill() {
  if (!join_pending_) return;
  check(cudaStreamWaitEvent(cur_, join_ev_, 0), "stream wait");
  join_pending_ = false;
}

double dt_inclusive(double tstart, double tstop, int L) {  // :224-237
  return (tstop - tstart) / (std::pow(2., L + 1) - 1);
}

// Polarization vector of src/OSCARSSR.cc:4116-4150 (host double arithmetic, reference order).
void polarization_vector(const osc_rad_opts& o, double P[6], bool& project) {
  const Vec3 hor = v3(o.horizontal[0], o.horizontal[1], o.horizontal[2]);
  const Vec3 prop = v3(o.propagation[0], o.propagation[1], o.propagation[2]);
  const Vec3 vert = unit(cross(prop, hor));
  const double k = 1. / std::sqrt(2);
  for (int i = 0; i < 6; ++i) P[i] = 0;
  switch (o.polarization) {
    case OSC_POL_ALL: break;
    case OSC_POL_LH: P[0] = hor.x; P[2] = hor.y; P[4] = hor.z; break;
    case OSC_POL_LV: P[0] = vert.x; P[2] = vert.y; P[4] = vert.z; break;
    case OSC_POL_LINEAR: {
      const Vec3 r = rotate_about(hor, o.angle, prop);
      P[0] = r.x; P[2] = r.y; P[4] = r.z;
      break;
    }
    case OSC_POL_CL:
    case OSC_POL_CR: {
      const double sg = o.polarization == OSC_POL_CL ? 1.0 : -1.0;
      const double h[3] = {hor.x, hor.y, hor.z}, v[3] = {vert.x, vert.y, vert.z};
      for (int c = 0; c < 3; ++c) {
        P[2 * c] = (sg > 0 ? h[c] + v[c] * 0 : h[c] - v[c] * 0) * k;
        P[2 * c + 1] = (sg > 0 ? 0 + v[c] * 1 : 0 - v[c] * 1) * k;
      }
      break;
    }
    default: throw Error{OSC_ERR_INVALID, "Polarization requested not recognized"};
  }
  const double m2 = (P[0] * P[0] + P[1] * P[1]) + (P[2] * P[2] + P[3] * P[3]) + (P[4] * P[4] + P[5] * P[5]);
  project = o.polarization != OSC_POL_ALL && m2 > 0.001;
}

// Levels resident before a request starts: every wave up to this level is enqueued without any
// host round trip; entries still unconverged after it make the host extend the cache.
constexpr int kPrefillLevel = 14;
constexpr int kMinSpan = 32;
// Sample-split flux / spectrum waves (FP64 and mixed): spans of at least one staged chunk, so that a
// unit's fixed costs (its first copy, the partial store, the tile counter) stay small beside its
// arithmetic.
constexpr int kMinSpanSplit = 128;

int Engine::wave_grid(int kind, int variant) {
  if (wave_grid_[kind][variant] == 0) {
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attr");
    const int per = kind == 2   ? mixed_blocks_per_sm(variant)
                    : kind == 4 ? pd_mixed_blocks_per_sm()
                                : fp64_blocks_per_sm(kind == 1, variant);
    wave_grid_[kind][variant] = sms * per;
  }
  return wave_grid_[kind][variant];
}

// Autotuner: the first request of a given shape (kind, size class, level range) runs the waves
// with every compiled variant of the sample-sum kernel into scratch outputs, times them with CUDA
// events, and keeps the fastest for that shape.  FP64 variants differ only in their register cap,
// so they give bit-identical sums; mixed variants also change entries per thread.
// Statistics of one request into its mapped pinned ring slot: not converged, samples, the sticky
// error word (read by collect() after the slot's event).
__device__ __forceinline__ void k_stats_store(const unsigned long long* __restrict__ c64,
                                              const unsigned* __restrict__ err, volatile unsigned long long* slot) {
  slot[0] = c64[0];
  slot[1] = c64[1];
  slot[2] = *err;
}

__global__ void k_stats_out(const unsigned long long* __restrict__ c64, const unsigned* __restrict__ err,
                            volatile unsigned long long* slot) {
  k_stats_store(c64, err, slot);
}

// Start of a request in one launch: zero up to three ranges of 32-bit words (the request's counters,
// the fused-finalize counters, the beta-step maxima of the levels to fill) and copy the frequencies
// from the mapped staging buffer.
struct ZeroRange {
  unsigned* p;
  int64_t words;
};
__global__ void k_request_prologue(ZeroRange z0, ZeroRange z1, ZeroRange z2, const double* __restrict__ om_src,
                                   double* __restrict__ om_dst, int64_t n_om) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t i = t0; i < z0.words; i += stride) z0.p[i] = 0u;
  for (int64_t i = t0; i < z1.words; i += stride) z1.p[i] = 0u;
  for (int64_t i = t0; i < z2.words; i += stride) z2.p[i] = 0u;
  for (int64_t i = t0; i < n_om; i += stride) om_dst[i] = om_src[i];
}

int Engine::pick_variant(int kind, RadRequest& rq, int64_t n_items, int Lfirst, int lstop, double* d_out,
                         int32_t* d_lvl, cudaStream_t st) {
  if (forced_variant[kind] >= 0) return forced_variant[kind];
  if (!autotune || tuning_ || kind == 1 || kind == 4) return current_variant_[kind];
  int lg = 0;
  while (((int64_t)1 << (lg + 1)) <= n_items) ++lg;
  const auto key = std::make_tuple(kind, lg, Lfirst, lstop);
  auto it = tuned_.find(key);
  if (it != tuned_.end()) return it->second;
  const int nvar = kind == 2 ? kMixedVariants : kFp64Variants;
  const bool prof = profiling;
  profiling = false;
  tuning_ = true;
  cudaEvent_t a, b;
  check(cudaEventCreate(&a), "event");
  check(cudaEventCreate(&b), "event");
  int best = current_variant_[kind];
  float best_ms = 1e30f;
  const long long saved_launches = last_launches;
  for (int v = 0; v < nvar; ++v) {
    current_variant_[kind] = v;
    run_single(rq, n_items, 1.0, d_out, d_lvl, st);  // warm (loads the module, fills caches)
    check(cudaEventRecord(a, st), "event");
    run_single(rq, n_items, 1.0, d_out, d_lvl, st);
    check(cudaEventRecord(b, st), "event");
    check(cudaEventSynchronize(b), "event");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, a, b), "event");
    if (ms < best_ms) { best_ms = ms; best = v; }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  pending_.clear();  // the statistics of the timing runs are not the request's
  last_launches = saved_launches;
  tuning_ = false;
  profiling = prof;
  current_variant_[kind] = best;
  tuned_[key] = best;
  return best;
}

void Engine::run_single(const RadRequest& rq, int64_t n_items, double weight, double* d_out, int32_t* d_lvl,
                        cudaStream_t st) {
  const osc_rad_opts& o = rq.opts;
  int ext_from = kMaxLevelMemory;
  const int lstop = request_levels(o, kMaxLevelExtendedGpu, &ext_from);
  set_level_grid(ext_from);
  const Particle& P = model.particle;
  const bool mixed = o.precision_mode == OSC_MIXED;
  const int Lfirst = std::min(9, lstop);
  const int kind = rq.power_density ? (mixed ? 4 : 1) : (mixed ? 2 : 0);
  // Levels enqueued without a host round trip: up to kPrefillLevel, or, for a request shape seen
  // before, up to the highest level its previous call needed (waves past it would find no entries;
  // levels beyond are still added by the host loop below when entries remain).
  const auto hist_key = std::make_tuple(kind, n_items, (int64_t)rq.omega.size(), lstop, o.precision);
  const auto hist = prefill_hist_.find(hist_key);
  const int Lpre_want = hist != prefill_hist_.end() ? hist->second : kPrefillLevel;
  const int Lpre = std::min(lstop, std::max(Lfirst, Lpre_want));
  const int variant = tuning_ ? current_variant_[kind]
                              : pick_variant(kind, const_cast<RadRequest&>(rq), n_items, Lfirst, lstop, d_out, d_lvl, st);
  const int resident = wave_grid(kind, variant);  // CTAs resident at once on the device
  const int tile = rq.power_density ? (mixed ? pd_mixed_entries_per_cta() : 128)
                                    : (mixed ? mixed_entries_per_cta(variant) : fp64_entries_per_cta(variant));
  const int min_span = rq.power_density ? kMinSpan : kMinSpanSplit;
  const int64_t target = 4 * (int64_t)resident;   // >= 4 waves of equal units per launch
  const int64_t N = n_items;
  // Partial-sum buffer: a wave has tiles x spans units with spans the smallest power of two reaching
  // the target (wave_spans), so tiles x spans < max(tiles, 2 x target) whatever the active count;
  // every unit stores 2 segments x `per` values for each of its `tile` entry slots.
  const int per = rq.power_density ? 1 : kFdPartials;
  const int64_t ntiles = (N + tile - 1) / tile;
  const size_t part_doubles = (size_t)2 * per * tile * std::max<int64_t>(ntiles, 2 * target);
  // Per-level grid: the largest unit count over the active counts the level can have, capped at the
  // resident CTAs.  The first wave has all N entries; a later wave with t tiles has t x spans units,
  // which reaches the target (> resident) once t x (largest span count of the level) does.
  auto grid_for = [&](int L) -> int {
    if (L == Lfirst) {
      const WavePlan pl = wave_plan(1, L, N, tile, target, min_span);
      return (int)std::min<int64_t>(pl.tiles * pl.spans, resident);
    }
    const int64_t span_max = wave_spans(L, 1, INT64_MAX, min_span);
    return (int)std::min<int64_t>(ntiles * span_max, resident);
  };
  part_.reserve(sizeof(double) * part_doubles);
  act_[0].reserve(sizeof(int) * N);
  act_[1].reserve(sizeof(int) * N);
  state_.reserve(sizeof(double) * 7 * N);

  unsigned* cnt = cnt_.as<unsigned>();  // [0], [1] list counts, [kCntErr] sticky error word
  // [0] not converged, [1] samples, [2] unit counter of the running wave
  unsigned long long* c64 = reinterpret_cast<unsigned long long*>(cnt + 4);
  unsigned* level_max = cnt + 12;  // highest level at which an entry finished
  // Flux / spectrum waves finalize their own tiles (one launch per level).  Wave w reads its active
  // count from fz3[w % 3], appends survivors to fz3[(w + 1) % 3] and zeroes fz3[(w + 2) % 3] for the
  // wave after; it takes units from fw[w % 2] and zeroes fw[(w + 1) % 2].
  const bool fused = !rq.power_density || mixed;  // the FP64 power density keeps its finalize kernel
  unsigned* fz3 = nullptr;
  unsigned long long* fw = nullptr;
  if (fused) {
    fused_.reserve(64 + sizeof(unsigned) * (size_t)(ntiles + 1));
    fz3 = fused_.as<unsigned>();
    fw = reinterpret_cast<unsigned long long*>(fz3 + 4);
  }
  // One prologue launch zeroes the counters (words 0..12), the fused-finalize counters and the
  // beta-step maxima of the levels the prefill fills, and copies the staged frequencies.
  {
    if (mixed) reserve_mixed(Lpre);
    else reserve_levels(Lpre);
    const int filled = mixed ? mrec_filled_ : lev_filled_;
    ZeroRange z0{cnt, 13}, z1{fz3, fused ? 16 + (ntiles + 1) : 0}, z2{nullptr, 0};
    if (Lpre > filled) {
      if (mixed) {
        const int Lb = filled < 0 ? 0 : filled + 1;
        z2 = ZeroRange{mrec_bd_.as<unsigned>() + 2 * Lb, 2 * (int64_t)(Lpre - Lb + 1)};
      } else if (filled < 0) {
        z2 = ZeroRange{bd_bits_.as<unsigned>(), 64};
      }
    }
    const int64_t n_om = omega_staged_;
    const int64_t words = std::max<int64_t>(std::max<int64_t>(z0.words, z1.words), std::max<int64_t>(z2.words, n_om));
    const int blocks = (int)std::min<int64_t>((words + 255) / 256, 148);
    k_request_prologue<<<blocks, 256, 0, st>>>(z0, z1, z2, stage_host_, omega_.as<double>(), n_om);
    check(cudaGetLastError(), "request prologue");
    ++last_launches;
    if (n_om > 0) {  // the staging buffer is free again once the prologue has run
      check(cudaEventRecord(stage_ev_, st), "event");
      omega_staged_ = 0;
    }
  }
  prefill(mixed, Lfirst, Lpre, true);

  const double* d_obs = req_obs_;
  const double* d_nrm = rq.normals ? req_nrm_ : nullptr;
  double pol[6];
  bool project = false;
  double c0 = 0, c2 = 0, scale = 0;
  if (!rq.power_density) {
    polarization_vector(o, pol, project);
    c0 = P.q / (four_pi() * kC * kEps0 * kSqrt2Pi);                                       // :4106
    const double cur = rq.spectrum_current_abs ? std::fabs(P.current) : P.current;
    c2 = four_pi() * cur / (kH * std::fabs(P.q) * kMu0 * kC) * 1e-6 * 0.001;              // :4109
    if (mixed) {  // project in the frame: P' = R P (R orthogonal, so E'.P' = E.P)
      double pr[6];
      const double* R = frame_.rot;
      for (int ri = 0; ri < 2; ++ri)
        for (int r = 0; r < 3; ++r)
          pr[2 * r + ri] = R[3 * r] * pol[ri] + R[3 * r + 1] * pol[2 + ri] + R[3 * r + 2] * pol[4 + ri];
      for (int i = 0; i < 6; ++i) pol[i] = pr[i];
    }
  } else {
    scale = std::fabs(P.q * P.current) / (16 * (kPi * kPi) * kEps0 * kC);                 // :2945
  }

  int cur_list = 0;
  auto launch_wave = [&](int L) {
    const bool first = L == Lfirst;
    if (first) wait_inputs(st);  // observers from the host
    else join_prefill();         // the levels filled on the side stream
    const int wv = L - Lfirst;
    const int* act_in = first ? nullptr : act_[cur_list].as<int>();
    const unsigned* nact_in = first ? nullptr : (fused ? fz3 + wv % 3 : cnt + cur_list);
    unsigned* n_next = fused ? fz3 + (wv + 1) % 3 : cnt + (cur_list ^ 1);
    if (!fused) check(cudaMemsetAsync(n_next, 0, sizeof(unsigned), st), "memset");
    if (fused && rq.power_density) {
      PdWaveArgs w{};
      w.lev = reinterpret_cast<const double*>(mrec_.p);
      w.cap = lev_cap_; w.obs = d_obs; w.normals = d_nrm; w.has_normal = d_nrm != nullptr;
      w.directional = rq.directional; w.n_items = N; w.act = act_in; w.n_act = nact_in;
      w.first = first; w.level = L; w.tile_entries = tile; w.min_span = min_span; w.target_units = target;
      w.part = part_.as<double>(); w.err = cnt + kCntErr; w.work = fw + wv % 2;
      w.fused = 1;
      w.tile_done = fz3 + 16;
      w.zero_u32 = fz3 + (wv + 2) % 3;
      w.zero_u64 = fw + (wv + 1) % 2;
      PdFinalArgs& f = w.fin;
      f.part = part_.as<double>(); f.first = first; f.level = L; f.max_level = lstop; f.quantity = o.quantity;
      f.directional = rq.directional; f.tile_entries = tile; f.min_span = min_span; f.target_units = target;
      f.dt_prev = L >= 1 ? dt_inclusive(tstart_, tstop_, L - 1) : 0; f.dt_level = dt_inclusive(tstart_, tstop_, L);
      f.precision = o.precision; f.scale = scale; f.weight = weight; f.two_over_gamma = 2. / P.gamma;
      f.bdmax_levels = reinterpret_cast<const double*>(mrec_bd_.p);
      f.n_items = N; f.act = act_in; f.n_act = nact_in; f.state = state_.as<double>();
      f.act_next = act_[cur_list ^ 1].as<int>(); f.n_next = n_next;
      f.out = d_out; f.level_out = d_lvl; f.not_converged = c64; f.samples = c64 + 1; f.level_max = level_max;
      f.work_reset = nullptr;
      auto ev = timed_begin(st);
      check(launch_pd_wave_mixed(w, frame_, grid_for(L), st), "power density wave (mixed)");
      timed_end(ev, st);
      last_launches += 1;
      cur_list ^= 1;
      return;
    }
    if (fused) {
      FdWaveArgs w{};
      w.lev = mixed ? reinterpret_cast<const double*>(mrec_.p) : lev_.as<double>();
      w.cap = lev_cap_; w.obs = d_obs; w.omega = omega_.as<double>();
      w.n_e = (int64_t)rq.omega.size(); w.n_items = N; w.act = act_in; w.n_act = nact_in;
      w.first = first; w.level = L; w.tile_entries = tile; w.min_span = min_span; w.target_units = target;
      w.part = part_.as<double>(); w.err = cnt + kCntErr; w.work = fw + wv % 2;
      w.fused = 1;
      w.tile_done = fz3 + 16;
      w.zero_u32 = fz3 + (wv + 2) % 3;
      w.zero_u64 = fw + (wv + 1) % 2;
      FdFinalArgs& f = w.fin;
      f.part = part_.as<double>(); f.first = first; f.level = L; f.max_level = lstop; f.quantity = o.quantity;
      f.project = project; f.tile_entries = tile; f.min_span = min_span; f.target_units = target;
      f.dt_prev = L >= 1 ? dt_inclusive(tstart_, tstop_, L - 1) : 0; f.dt_level = dt_inclusive(tstart_, tstop_, L);
      f.precision = o.precision; f.c0 = c0; f.c2 = c2; f.weight = weight;
      for (int i = 0; i < 6; ++i) f.pol[i] = pol[i];
      f.n_items = N; f.act = act_in; f.n_act = nact_in; f.state = state_.as<double>();
      f.act_next = act_[cur_list ^ 1].as<int>(); f.n_next = n_next;
      f.out = d_out; f.level_out = d_lvl; f.not_converged = c64; f.samples = c64 + 1; f.level_max = level_max; f.work_reset = nullptr;
      f.dmax_spans_joined = 1;  // the flux waves carry the step into each part across groups and spans
      auto ev = timed_begin(st);
      const int g = grid_for(L);
      if (mixed) check(launch_fd_wave_mixed(w, frame_, g, variant, st), "flux wave (mixed)");
      else check(launch_fd_wave_fp64(w, g, variant, st), "flux wave");
      timed_end(ev, st);
      last_launches += 1;
      cur_list ^= 1;
      return;
    }
    if (!rq.power_density) {
      FdWaveArgs w{};
      w.lev = mixed ? reinterpret_cast<const double*>(mrec_.p) : lev_.as<double>();
      w.cap = lev_cap_; w.obs = d_obs; w.omega = omega_.as<double>();
      w.n_e = (int64_t)rq.omega.size(); w.n_items = N; w.act = act_in; w.n_act = nact_in;
      w.first = first; w.level = L; w.tile_entries = tile; w.min_span = min_span; w.target_units = target;
      w.part = part_.as<double>(); w.err = cnt + kCntErr; w.work = c64 + 2;
      auto ev = timed_begin(st);
      const int g = grid_for(L);
      if (mixed) check(launch_fd_wave_mixed(w, frame_, g, variant, st), "flux wave (mixed)");
      else check(launch_fd_wave_fp64(w, g, variant, st), "flux wave");
      timed_end(ev, st);
      FdFinalArgs f{};
      f.part = part_.as<double>(); f.first = first; f.level = L; f.max_level = lstop; f.quantity = o.quantity;
      f.project = project; f.tile_entries = tile; f.min_span = min_span; f.target_units = target;
      f.dt_prev = L >= 1 ? dt_inclusive(tstart_, tstop_, L - 1) : 0; f.dt_level = dt_inclusive(tstart_, tstop_, L);
      f.precision = o.precision; f.c0 = c0; f.c2 = c2; f.weight = weight;
      for (int i = 0; i < 6; ++i) f.pol[i] = pol[i];
      f.n_items = N; f.act = act_in; f.n_act = nact_in; f.state = state_.as<double>();
      f.act_next = act_[cur_list ^ 1].as<int>(); f.n_next = n_next;
      f.out = d_out; f.level_out = d_lvl; f.not_converged = c64; f.samples = c64 + 1; f.level_max = level_max; f.work_reset = c64 + 2;
      check(launch_fd_finalize(f, N, st), "flux finalize");
    } else {
      PdWaveArgs w{};
      w.lev = mixed ? reinterpret_cast<const double*>(mrec_.p) : lev_.as<double>();
      w.cap = lev_cap_; w.obs = d_obs; w.normals = d_nrm; w.has_normal = d_nrm != nullptr;
      w.directional = rq.directional; w.n_items = N; w.act = act_in; w.n_act = nact_in;
      w.first = first; w.level = L; w.tile_entries = tile; w.min_span = min_span; w.target_units = target;
      w.part = part_.as<double>(); w.err = cnt + kCntErr; w.work = c64 + 2;
      auto ev = timed_begin(st);
      if (mixed) check(launch_pd_wave_mixed(w, frame_, grid_for(L), st), "power density wave (mixed)");
      else check(launch_pd_wave_fp64(w, grid_for(L), st), "power density wave");
      timed_end(ev, st);
      PdFinalArgs f{};
      f.part = part_.as<double>(); f.first = first; f.level = L; f.max_level = lstop; f.quantity = o.quantity;
      f.directional = rq.directional; f.tile_entries = tile; f.min_span = min_span; f.target_units = target;
      f.dt_prev = L >= 1 ? dt_inclusive(tstart_, tstop_, L - 1) : 0; f.dt_level = dt_inclusive(tstart_, tstop_, L);
      f.precision = o.precision; f.scale = scale; f.weight = weight; f.two_over_gamma = 2. / P.gamma;
      f.bdmax_levels = reinterpret_cast<const double*>(mixed ? mrec_bd_.p : bd_bits_.p);
      f.n_items = N; f.act = act_in; f.n_act = nact_in; f.state = state_.as<double>();
      f.act_next = act_[cur_list ^ 1].as<int>(); f.n_next = n_next;
      f.out = d_out; f.level_out = d_lvl; f.not_converged = c64; f.samples = c64 + 1; f.level_max = level_max; f.work_reset = c64 + 2;
      check(launch_pd_finalize(f, N, st), "power density finalize");
    }
    last_launches += 2;
    cur_list ^= 1;
  };
  for (int L = Lfirst; L <= Lpre; ++L) launch_wave(L);
  bool finished = false;  // statistics (and result downloads) already enqueued behind the last wave
  for (int L = Lpre + 1; L <= lstop; ++L) {  // beyond the prefilled levels the host decides
    // a one-thread kernel writes the active count and the highest finished level into mapped host
    // memory behind a sequence word that the host polls (no copy engine, no stream wake-up)
    const unsigned* active = fused ? fz3 + (L - Lfirst) % 3 : cnt + cur_list;
    unsigned nn = 0, lmax = 0;
    // the report also stores the request's statistics into a ring slot, and the downloads of host
    // outputs go in behind it, before the host knows whether this was the last wave; if it was not,
    // both are superseded by those the request ends with
    const bool speculate = !tuning_;
    const int slot = speculate ? claim_stat_slot() : -1;
    const unsigned seq = report_launch(active, level_max, st, speculate ? c64 : nullptr,
                                       speculate ? stats_host_ + kStatWords * slot : nullptr);
    if (speculate) finish_request(slot, st);
    report_wait(seq, &nn, &lmax, st);
    if (nn == 0) {
      if (!tuning_) prefill_hist_[hist_key] = std::max<int>(Lfirst, (int)lmax);
      finished = speculate;
      break;
    }
    if (speculate) {
      pending_.pop_back();
      tail_.emitted = false;
    }
    if (mixed) ensure_mixed(L);
    else ensure_levels(L);
    launch_wave(L);
  }
  join_prefill();
  wait_inputs(st);  // no upload into the request's buffers stays in flight past the request
  if (!finished) {
    const int slot = claim_stat_slot();
    k_stats_out<<<1, 1, 0, st>>>(c64, cnt_.as<unsigned>() + kCntErr, stats_host_ + kStatWords * slot);
    check(cudaGetLastError(), "stats");
    ++last_launches;
    finish_request(slot, st);
  }
}

int Engine::claim_stat_slot() {
  if ((int)pending_.size() >= kStatSlots) collect();
  return stats_slot_++ % kStatSlots;
}

// The statistics of the request just enqueued, stored into ring slot `slot` by the last kernel on
// the stream, are read by collect() when asked (after the slot's event); a single-particle request
// with host outputs then enqueues its result downloads.
void Engine::finish_request(int slot, cudaStream_t st) {
  check(cudaEventRecord(stats_ev_[slot], st), "event");
  pending_.push_back(slot);
  if (!tail_.active || tuning_) return;
  check(cudaMemcpyAsync(tail_.h_out, tail_.d_out, sizeof(double) * tail_.n, cudaMemcpyDeviceToHost, st), "download");
  if (tail_.h_lvl)
    check(cudaMemcpyAsync(tail_.h_lvl, tail_.d_lvl, sizeof(int32_t) * tail_.n, cudaMemcpyDeviceToHost, st),
          "download");
  tail_.emitted = true;
}

void Engine::wait_inputs(cudaStream_t st) {
  if (!inputs_pending_) return;
  check(cudaStreamWaitEvent(st, in_ev_, 0), "stream wait");
  inputs_pending_ = false;
}

// Wait for the statistics of the enqueued particles of the last request and report device errors.
void Engine::collect() {
  if (device < 0) return;
  // the error word rides in the slots (the last one has every earlier error: the word is sticky);
  // with no slot pending it is read directly
  unsigned err = 0;
  const bool direct = pending_.empty();
  for (int slot : pending_) {
    check(cudaEventSynchronize(stats_ev_[slot]), "radiation");
    const volatile unsigned long long* w = stats_host_ + kStatWords * slot;
    last_not_converged += (long long)w[0];
    last_samples += (long long)w[1];
    err |= (unsigned)w[2];
    if (profiling) prof_samples += (long long)w[1];
  }
  pending_.clear();
  if (profiling) collect_timings();
  if (direct) check(cudaMemcpy(&err, cnt_.as<unsigned>() + kCntErr, sizeof err, cudaMemcpyDeviceToHost), "error word");
  if (err) {
    check(cudaMemset(cnt_.as<unsigned>() + kCntErr, 0, sizeof(unsigned)), "error word");
    if (err & 1u) throw Error{OSC_ERR_TIMEOUT, "a staged trajectory copy did not complete (device wait limit reached)"};
    if (err & 8u) throw Error{OSC_ERR_STATE, "a sample-sum kernel variant was planned with another tile size"};
    throw Error{OSC_ERR_INVALID, kMixedGeometryMessage};
  }
}

// Make `s` the stream of the work that follows.  The caches (trajectory, level samples, records) and
// the request scratch are shared by all requests of the context, so when the stream changes, `s`
// first waits for everything enqueued on the previous one.
void Engine::use_stream(cudaStream_t s) {
  if (last_stream_valid_ && last_stream_ != s) {
    check(cudaEventRecord(order_ev_, last_stream_), "event");
    check(cudaStreamWaitEvent(s, order_ev_, 0), "stream wait");
  }
  last_stream_ = s;
  last_stream_valid_ = true;
  cur_ = s;
}

// Trajectories of a list of particles integrated on host worker threads ahead of their use: worker
// threads claim particles in order and fill a ring of slots; the consumer takes particle k's slot
// when it is ready and releases it for particle k + slots.  A worker's exception is rethrown to
// the consumer at that particle.
class TrajectoryPipeline {
 public:
  // `device`: the workers also lay each trajectory out in pinned host memory in the device knot
  // layout (t | y[9] | ypp[9] | diag), so that its upload is one asynchronous copy.
  // `pool`: pinned staging buffers and their copy events, kept by the engine between requests (pinned
  // allocations are slow); grown here to the slots this pipeline uses.
  TrajectoryPipeline(const Model& m, const std::vector<Particle>& parts, int device, std::vector<PinnedStage>& pool)
      : m_(m), parts_(parts), device_(device) {
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    const int nthreads = (int)std::min<size_t>(std::min(hw - 1u, 32u), std::max<size_t>(1, parts.size()));
    const size_t nslots = std::min<size_t>(2 * nthreads, std::max<size_t>(1, parts.size()));
    while (pool.size() < nslots) {
      pool.emplace_back();
      const cudaError_t e = cudaEventCreateWithFlags(&pool.back().copied, cudaEventDisableTiming);
      if (e != cudaSuccess) throw Error{OSC_ERR_CUDA, std::string("event: ") + cudaGetErrorString(e)};
    }
    slots_.resize(nslots);
    for (size_t i = 0; i < nslots; ++i) slots_[i].stage = &pool[i];
    for (int i = 0; i < nthreads; ++i) workers_.emplace_back([this] { work(); });
  }
  ~TrajectoryPipeline() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  // The upload of particle k's pinned copy was enqueued on `st`: the slot's next trajectory is staged
  // only after that copy has run (the request need not have waited for the device by then).
  void uploaded(size_t k, cudaStream_t st) {
    const cudaError_t e = cudaEventRecord(slots_[k % slots_.size()].stage->copied, st);
    if (e != cudaSuccess) throw Error{OSC_ERR_CUDA, std::string("event: ") + cudaGetErrorString(e)};
  }
  // Particle k's trajectory: its knots and their pinned copy in the device layout.  The slot stays
  // the caller's until release(k), so the copy may still be read by the device until then.
  Knots& wait(size_t k, const double** pinned) {
    Slot& s = slots_[k % slots_.size()];
    std::unique_lock<std::mutex> g(mu_);
    cv_.wait(g, [&] { return s.ready && s.particle == (int64_t)k; });
    if (s.err) std::rethrow_exception(s.err);
    *pinned = s.stage->pinned;
    return s.knots;
  }
  void release(size_t k) {
    {
      std::lock_guard<std::mutex> g(mu_);
      slots_[k % slots_.size()].ready = false;
      consumed_ = k + 1;
    }
    cv_.notify_all();
  }

 private:
  struct Slot {
    Knots knots;
    std::vector<double> sweep[2];
    PinnedStage* stage = nullptr;
    int64_t particle = -1;
    bool ready = false;
    std::exception_ptr err;
  };
  static void stage(Slot& s, int device) {  // knots -> pinned t | y | ypp | diag
    const Knots& k = s.knots;
    PinnedStage& p = *s.stage;
    const size_t n = (size_t)k.n, need = 20 * n;
    cudaError_t ev = cudaEventSynchronize(p.copied);  // the previous copy out of this buffer has run
    if (ev != cudaSuccess) throw Error{OSC_ERR_CUDA, std::string("event: ") + cudaGetErrorString(ev)};
    if (p.doubles < need) {
      if (p.pinned) cudaFreeHost(p.pinned);
      p.pinned = nullptr;
      p.doubles = 0;
      cudaError_t e = cudaSetDevice(device);
      if (e == cudaSuccess)
        e = cudaHostAlloc(reinterpret_cast<void**>(&p.pinned), sizeof(double) * need, cudaHostAllocPortable);
      if (e != cudaSuccess) throw Error{OSC_ERR_CUDA, std::string("cudaHostAlloc: ") + cudaGetErrorString(e)};
      p.doubles = need;
    }
    std::memcpy(p.pinned, k.t.data(), sizeof(double) * n);
    std::memcpy(p.pinned + n, k.y.data(), sizeof(double) * 9 * n);
    std::memcpy(p.pinned + 10 * n, k.ypp.data(), sizeof(double) * 9 * n);
    if (k.diag.size() == n) std::memcpy(p.pinned + 19 * n, k.diag.data(), sizeof(double) * n);
    else std::memset(p.pinned + 19 * n, 0, sizeof(double) * n);
  }
  void work() {
    for (;;) {
      size_t k;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || next_ >= parts_.size() || next_ < consumed_ + slots_.size(); });
        if (stop_ || next_ >= parts_.size()) return;
        k = next_++;
      }
      Slot& s = slots_[k % slots_.size()];
      std::exception_ptr err;
      try {
        m_.integrate(parts_[k], s.knots, s.sweep, false);
        stage(s, device_);
      } catch (...) {
        err = std::current_exception();
      }
      {
        std::lock_guard<std::mutex> g(mu_);
        s.err = err;
        s.particle = (int64_t)k;
        s.ready = true;
      }
      cv_.notify_all();
    }
  }
  const Model& m_;
  const std::vector<Particle>& parts_;
  const int device_;
  std::vector<Slot> slots_;
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_;
  size_t next_ = 0, consumed_ = 0;
  bool stop_ = false;
};

__global__ void k_report_counts(const unsigned* __restrict__ a, const unsigned* __restrict__ b,
                                volatile unsigned* host, unsigned seq, const unsigned long long* __restrict__ c64,
                                const unsigned* __restrict__ err, volatile unsigned long long* slot) {
  if (slot) k_stats_store(c64, err, slot);
  host[1] = *a;
  host[2] = *b;
  __threadfence_system();
  host[0] = seq;
}

// The two device words `a` and `b` once the stream reaches this point: a one-thread kernel stores
// them into the mapped control words (ctl_host_[1], [2]) and then the sequence number into [0],
// which the host polls; every 4096 polls it asks whether the stream has finished, so a failed or
// lost launch ends in the stream's error instead of a wait that does not end.
void Engine::report_counts(const unsigned* a, const unsigned* b, unsigned* va, unsigned* vb, cudaStream_t st) {
  report_wait(report_launch(a, b, st), va, vb, st);
}

unsigned Engine::report_launch(const unsigned* a, const unsigned* b, cudaStream_t st, const unsigned long long* c64,
                               unsigned long long* slot) {
  const unsigned seq = ++report_seq_;
  k_report_counts<<<1, 1, 0, st>>>(a, b, ctl_host_, seq, c64, cnt_.as<unsigned>() + kCntErr, slot);
  check(cudaGetLastError(), "count");
  ++last_launches;
  return seq;
}

void Engine::report_wait(unsigned seq, unsigned* va, unsigned* vb, cudaStream_t st) {
  volatile unsigned* w = ctl_host_;
  for (unsigned i = 1; w[0] != seq; ++i) {
    if ((i & 4095u) == 0) {
      const cudaError_t e = cudaStreamQuery(st);
      if (e != cudaErrorNotReady) {
        check(e, "count");
        if (w[0] != seq) throw Error{OSC_ERR_CUDA, "count: the report kernel did not write its sequence number"};
      }
    }
  }
  *va = w[1];
  *vb = w[2];
}

void Engine::radiation(RadRequest& rq) {
  if (device < 0) throw Error{OSC_ERR_NO_DEVICE, "this context was created without a GPU (device -1)"};
  check(cudaSetDevice(device), "cudaSetDevice");
  use_stream(rq.stream ? rq.stream : stream);
  // statistics describe the latest request: drop those of earlier ones without waiting for them
  // (their ring slots may be rewritten; copies into a slot stay in stream order)
  pending_.clear();
  last_samples = last_launches = last_not_converged = 0;
  cudaStream_t st = rq.stream ? rq.stream : stream;
  const int64_t n_e = rq.power_density ? 1 : (int64_t)rq.omega.size();
  const int64_t N = rq.n_obs * n_e;
  if (N <= 0) return;
  if (N > 2147483647ll) throw Error{OSC_ERR_LENGTH, "more than 2^31-1 (observer, energy) entries in one call"};
  // Inputs.  Device observers (and normals) are read where they are.  Host ones go up on copy_ (after
  // the work already on the request stream, which may still read the previous request's uploads),
  // concurrently with the level samples the request stream builds; the first wave waits for them
  // (wait_inputs).  (Reading page-locked observers in place over PCIe instead made the first wave
  // slower than the upload it saves.)  Up to kStageDoubles frequencies are staged in mapped
  // page-locked memory for the request prologue to copy; more go up directly.
  const int np = rq.opts.nparticles;
  if (rq.obs_on_device) {
    req_obs_ = rq.obs;
    req_nrm_ = rq.normals;
  } else {
    check(cudaEventRecord(in_fork_ev_, st), "event");
    check(cudaStreamWaitEvent(copy_, in_fork_ev_, 0), "stream wait");
    obs_.reserve(sizeof(double) * 3 * rq.n_obs);
    check(cudaMemcpyAsync(obs_.p, rq.obs, sizeof(double) * 3 * rq.n_obs, cudaMemcpyHostToDevice, copy_), "obs");
    if (rq.normals) {
      nrm_.reserve(sizeof(double) * 3 * rq.n_obs);
      check(cudaMemcpyAsync(nrm_.p, rq.normals, sizeof(double) * 3 * rq.n_obs, cudaMemcpyHostToDevice, copy_),
            "normals");
    }
    check(cudaEventRecord(in_ev_, copy_), "event");
    inputs_pending_ = true;
    req_obs_ = obs_.as<double>();
    req_nrm_ = rq.normals ? nrm_.as<double>() : nullptr;
  }
  omega_staged_ = 0;
  if (!rq.power_density) {
    omega_.reserve(sizeof(double) * n_e);
    if (n_e <= kStageDoubles) {
      check(cudaEventSynchronize(stage_ev_), "stage");
      std::memcpy(stage_host_, rq.omega.data(), sizeof(double) * n_e);
      omega_staged_ = n_e;
    } else {
      check(cudaMemcpyAsync(omega_.p, rq.omega.data(), sizeof(double) * n_e, cudaMemcpyHostToDevice, st), "omega");
    }
  }
  out_.reserve(sizeof(double) * N);
  lvl_.reserve(sizeof(int32_t) * N);
  double* d_out = rq.out_on_device ? rq.out : out_.as<double>();
  int32_t* d_lvl = rq.out_on_device ? rq.level_out : lvl_.as<int32_t>();
  if (!d_lvl) d_lvl = lvl_.as<int32_t>();
  // Host outputs are downloaded by the copy engine right behind the last report (ResultTail).
  // (Kernel stores straight into mapped page-locked outputs were measured too: a few microseconds
  // faster on one box and tens slower on another, so the copies are kept.)

  // Mixed multi-particle flux / spectrum requests with at least beam_batch_min particles (this
  // process's share) run as one batch with device RK4 trajectories; smaller ones, and those with RKAS
  // trajectories, take the host integrator on worker threads like the FP64 path: the device RK4 is a
  // serial chain per particle (~4 us per step, ~60 ms for 16001 points whatever the batch size), which
  // only pays once the batch is large.
  const int shard_n = rq.opts.shard_count > 1 ? rq.opts.shard_count : 1;
  const int shard_r = shard_n > 1 ? rq.opts.shard_rank % shard_n : 0;
  const int np_local = np > shard_r ? (np - shard_r + shard_n - 1) / shard_n : 0;
  if (np > 0 && rq.opts.precision_mode == OSC_MIXED && !rq.power_density && model.traj_method == Model::kRK4 &&
      np_local >= beam_batch_min) {
    radiation_beam_mixed(rq, N);
    return;
  }
  if (np <= 0) {
    model.ensure_trajectory();
    upload_trajectory();
    tail_ = ResultTail{};
    if (!rq.out_on_device) tail_ = ResultTail{true, false, d_out, d_lvl, rq.out, rq.level_out, N};
    try {
      run_single(rq, N, 1.0, d_out, d_lvl, st);
    } catch (...) {
      tail_ = ResultTail{};
      throw;
    }
    tail_.active = false;
  } else {
    // src/OSCARSSR.cc:4026-4062: new random particle, its trajectory, weight 1/N, compensated sum
    const double weight = 1.0 / (double)np;
    acc_.reserve(sizeof(double) * N);
    acc_comp_.reserve(sizeof(double) * N);
    check(cudaMemsetAsync(acc_.p, 0, sizeof(double) * N, st), "memset");
    check(cudaMemsetAsync(acc_comp_.p, 0, sizeof(double) * N, st), "memset");
    const int shards = rq.opts.shard_count > 1 ? rq.opts.shard_count : 1;
    std::vector<Particle> mine;  // this process's particles, drawn in the reference's order
    for (int ip = 0; ip < np; ++ip) {
      model.random_particle();
      if (ip % shards != rq.opts.shard_rank % shards) continue;  // another process's particle
      mine.push_back(model.particle);
    }
    {
      // their trajectories are integrated on host worker threads while the GPU sums earlier ones;
      // the model holds the particle in use and its trajectory (the last ones when done, as the
      // reference leaves them)
      TrajectoryPipeline pipe(model, mine, device, pin_pool_);
      for (size_t k = 0; k < mine.size(); ++k) {
        const double* pinned = nullptr;
        Knots& kn = pipe.wait(k, &pinned);
        model.particle = mine[k];
        std::swap(model.knots, kn);
        ++model.knots_version;
        upload_trajectory(pinned);
        pipe.uploaded(k, cur_);
        run_single(rq, N, weight, out_.as<double>(), d_lvl, st);
        pipe.release(k);
        k_kahan_add<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(acc_.as<double>(), acc_comp_.as<double>(),
                                                                  out_.as<double>(), N);
        check(cudaGetLastError(), "accumulate");
        ++last_launches;
      }
    }
    check(cudaMemcpyAsync(d_out, acc_.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, st), "result");
  }
  if (!rq.out_on_device) {
    if (!tail_.emitted) {  // (run_single enqueues them itself for one particle)
      check(cudaMemcpyAsync(rq.out, d_out, sizeof(double) * N, cudaMemcpyDeviceToHost, st), "download");
      if (rq.level_out)
        check(cudaMemcpyAsync(rq.level_out, d_lvl, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, st), "download");
    }
    tail_ = ResultTail{};
    check(cudaStreamSynchronize(st), "download");
    collect();
  }
}

// Multi-particle flux / spectrum in mixed precision: the particles are drawn on the host in the
// reference's order (src/OSCARSSR.cc:4026-4062) and integrated as one batch whose results are
// averaged with weight 1/N in particle order.
void Engine::radiation_beam_mixed(RadRequest& rq, int64_t N) {
  const int np = rq.opts.nparticles;
  const int64_t n_e = (int64_t)rq.omega.size();
  std::vector<double> obs_h;
  const double* obs = rq.obs;
  if (rq.obs_on_device) {
    obs_h.resize(3 * rq.n_obs);
    check(cudaMemcpy(obs_h.data(), rq.obs, sizeof(double) * 3 * rq.n_obs, cudaMemcpyDeviceToHost), "observers");
    obs = obs_h.data();
  }
  const int shards = rq.opts.shard_count > 1 ? rq.opts.shard_count : 1;
  std::vector<BatchJob> jobs;
  jobs.reserve(np / shards + 1);
  for (int ip = 0; ip < np; ++ip) {
    model.random_particle();
    if (ip % shards != rq.opts.shard_rank % shards) continue;  // another process's particle
    jobs.emplace_back();
    BatchJob& J = jobs.back();
    J.field_begin = 0;
    J.field_count = (int)model.fields.size();
    J.particle = model.particle;
    J.ctstart = model.ctstart;
    J.ctstop = model.ctstop;
    J.npoints = model.npoints;
    J.obs_begin = 0;
    J.n_obs = rq.n_obs;
    J.omega_begin = 0;
    J.n_e = n_e;
    J.current_abs = rq.spectrum_current_abs;
  }
  // the host trajectory now belongs to an earlier particle: recompute it on demand
  model.knots.clear();
  ++model.knots_version;
  std::vector<double> out_h, lvl_unused;
  std::vector<int32_t> lvl_h;
  double* out = rq.out;
  int32_t* lvl = rq.level_out;
  if (rq.out_on_device) {
    out_h.resize(N);
    lvl_h.resize(N);
    out = out_h.data();
    lvl = lvl_h.data();
  }
  if (jobs.empty()) {  // this shard has no particle: its share of the sum is zero
    std::fill(out, out + N, 0.0);
    if (lvl) std::fill(lvl, lvl + N, -1);
  } else {
    batch(model.fields, jobs, obs, rq.n_obs, rq.omega.data(), n_e, rq.opts, true, out, lvl, 1.0 / (double)np);
  }
  if (rq.out_on_device) {
    check(cudaMemcpy(rq.out, out_h.data(), sizeof(double) * N, cudaMemcpyHostToDevice), "result");
    if (rq.level_out)
      check(cudaMemcpy(rq.level_out, lvl_h.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice), "result");
  }
}

void Engine::batch_fp64(const std::vector<FieldSpec>& fields, const std::vector<BatchJob>& jobs, const double* obs,
                        int64_t n_obs_total, const double* omega, int64_t n_omega_total, const osc_rad_opts& o,
                        bool average, double* out, int32_t* level_out) {
  const int64_t m_avg = jobs.empty() ? 0 : jobs[0].n_obs * jobs[0].n_e;
  for (const BatchJob& J : jobs) {
    if (J.field_begin < 0 || J.field_count < 0 || (size_t)J.field_begin + J.field_count > fields.size())
      throw Error{OSC_ERR_RANGE, "job field range outside the field array"};
    if (J.obs_begin < 0 || J.n_obs < 1 || J.obs_begin + J.n_obs > n_obs_total)
      throw Error{OSC_ERR_RANGE, "job observer range outside the observer array"};
    if (J.omega_begin < 0 || J.n_e < 1 || J.omega_begin + J.n_e > n_omega_total)
      throw Error{OSC_ERR_RANGE, "job energy range outside the energy array"};
    if (average && (J.obs_begin != jobs[0].obs_begin || J.n_obs != jobs[0].n_obs ||
                    J.omega_begin != jobs[0].omega_begin || J.n_e != jobs[0].n_e))
      throw Error{OSC_ERR_INVALID, "averaged jobs must share their observers and energies"};
  }
  if (device < 0) throw Error{OSC_ERR_NO_DEVICE, "this context was created without a GPU (device -1)"};
  // the context's own model is set aside and restored; its trajectory is uploaded again afterwards
  Model saved = model;
  long long samples = 0, launches = 0, nnc = 0;
  std::vector<double> val, acc(average ? m_avg : 0, 0.0), comp(average ? m_avg : 0, 0.0);
  int64_t done = 0;
  try {
    for (size_t k = 0; k < jobs.size(); ++k) {
      const BatchJob& J = jobs[k];
      model.fields.assign(fields.begin() + J.field_begin, fields.begin() + J.field_begin + J.field_count);
      model.particle = J.particle;
      model.ctstart = J.ctstart;
      model.ctstop = J.ctstop;
      model.npoints = J.npoints;
      model.compute_trajectory();
      RadRequest rq;
      rq.obs = obs + 3 * J.obs_begin;
      rq.n_obs = J.n_obs;
      rq.omega.assign(omega + J.omega_begin, omega + J.omega_begin + J.n_e);
      rq.opts = o;
      rq.opts.nparticles = 0;
      rq.spectrum_current_abs = J.current_abs;
      const int64_t m = J.n_obs * J.n_e;
      if (average) {
        val.resize(m);
        rq.out = val.data();
        rq.level_out = (level_out && k + 1 == jobs.size()) ? level_out : nullptr;
      } else {
        rq.out = out + done;
        rq.level_out = level_out ? level_out + done : nullptr;
      }
      radiation(rq);
      samples += last_samples;
      launches += last_launches;
      nnc += last_not_converged;
      if (average) {  // compensated sum with weight 1/N in job order (T3DScalarContainer::AddToPoint)
        const double w = 1.0 / (double)jobs.size();
        for (int64_t i = 0; i < m; ++i) {
          const double y = val[i] * w - comp[i];
          const double t = acc[i] + y;
          comp[i] = (t - acc[i]) - y;
          acc[i] = t;
        }
      }
      done += m;
    }
  } catch (...) {
    const uint64_t v = model.knots_version;
    model = saved;
    model.knots_version = v + 1;
    throw;
  }
  const uint64_t v = model.knots_version;
  model = saved;
  model.knots_version = v + 1;  // a version no cached upload has seen
  if (average) std::copy(acc.begin(), acc.end(), out);
  last_samples = samples;
  last_launches = launches;
  last_not_converged = nnc;
}

std::pair<cudaEvent_t, cudaEvent_t> Engine::timed_begin(cudaStream_t st) {
  if (!profiling) return {nullptr, nullptr};
  auto get = [&]() {
    cudaEvent_t e;
    if (!ev_pool_.empty()) { e = ev_pool_.back(); ev_pool_.pop_back(); }
    else check(cudaEventCreate(&e), "cudaEventCreate");
    return e;
  };
  std::pair<cudaEvent_t, cudaEvent_t> e{get(), get()};
  check(cudaEventRecord(e.first, st), "cudaEventRecord");
  return e;
}

void Engine::timed_end(std::pair<cudaEvent_t, cudaEvent_t> e, cudaStream_t st) {
  if (!e.first) return;
  check(cudaEventRecord(e.second, st), "cudaEventRecord");
  ev_pending_.push_back(e);
}

void Engine::collect_timings() {
  for (auto& e : ev_pending_) {
    check(cudaEventSynchronize(e.second), "cudaEventSynchronize");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, e.first, e.second), "cudaEventElapsedTime");
    prof_ms += ms;
    ++prof_launches;
    ev_pool_.push_back(e.first);
    ev_pool_.push_back(e.second);
  }
  ev_pending_.clear();
}

namespace {
// FMA-throughput probe: 8 independent chains per thread, long enough that launch cost vanishes.
template <class T>
__global__ void k_fma_peak(T* out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = (T)(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = x[k] * a + b;
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == (T)-1.2345) out[threadIdx.x] = s;  // keeps the chains live
}
}  // namespace

double Engine::measure_fma_peak(int kind) {
  if (device < 0) throw Error{OSC_ERR_NO_DEVICE, "this context was created without a GPU (device -1)"};
  check(cudaSetDevice(device), "cudaSetDevice");
  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attr");
  out_.reserve(4096 * sizeof(double));
  const int threads = 256, blocks = sms * 8, iters = kind == 0 ? 4096 : 16384;
  cudaEvent_t a, b;
  check(cudaEventCreate(&a), "event");
  check(cudaEventCreate(&b), "event");
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    check(cudaEventRecord(a, stream), "event");
    if (kind == 0) k_fma_peak<double><<<blocks, threads, 0, stream>>>(out_.as<double>(), iters, 0.999999, 1e-7);
    else k_fma_peak<float><<<blocks, threads, 0, stream>>>(out_.as<float>(), iters, 0.999999f, 1e-7f);
    check(cudaGetLastError(), "fma peak");
    check(cudaEventRecord(b, stream), "event");
    check(cudaEventSynchronize(b), "event");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, a, b), "event");
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  const double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
  return flops / (best * 1e-3) / 1e12;
}

}  // namespace osc
