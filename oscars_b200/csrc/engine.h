// engine.h -- per-context device state and the wave scheduler of the radiation integrals.
#pragma once

#include <cstdint>
#include <string>
#include <map>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/oscars_b200.h"
#include "batch.h"
#include "host_core.h"
#include "kernels.h"

namespace osc {

// Device buffer that only grows.
// Highest level a flux, spectrum or power-density request may reach: levels above 26 (the reference's
// extended levels) are held in device memory like the others (2^(L+1) samples of 80 bytes, FP64; 72
// bytes, mixed), so a request is bounded by the free memory; the reference's own point count of a
// level is an int, which caps it at 30.
constexpr int kMaxLevelExtendedGpu = 30;
int request_levels(const osc_rad_opts& o, int max_supported, int* ext_from);

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void reserve(size_t n);
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

struct RadRequest {
  // frequency domain: entries = n_obs x n_e ; power density: entries = n_obs
  bool power_density = false;
  const double* obs = nullptr;      // 3*n_obs
  const double* normals = nullptr;  // 3*n_obs or NULL
  int64_t n_obs = 0;
  std::vector<double> omega;        // n_e angular frequencies
  bool obs_on_device = false;
  bool directional = false;
  osc_rad_opts opts{};
  bool spectrum_current_abs = false;  // spectrum uses |I| in C2 (src/OSCARSSR.cc:1888)
  double* out = nullptr;            // n_items
  int32_t* level_out = nullptr;
  bool out_on_device = false;
  cudaStream_t stream = nullptr;
};

// One job of a batch (host side): a particle with its trajectory range through fields
// [field_begin, field_begin + field_count) of the batch, observed at observers
// [obs_begin, obs_begin + n_obs) and energies [omega_begin, omega_begin + n_e) of the batch.
struct BatchJob {
  int field_begin = 0, field_count = 0;
  Particle particle;
  double ctstart = 0, ctstop = 0;
  int64_t npoints = 0;
  int64_t obs_begin = 0, n_obs = 0, omega_begin = 0, n_e = 0;
  bool current_abs = false;  // spectrum: |I| in the flux constant (src/OSCARSSR.cc:1888)
};

double dt_inclusive(double tstart, double tstop, int L);
void polarization_vector(const osc_rad_opts& o, double P[6], bool& project);

// A pinned host buffer for staging one trajectory's upload, with the event recorded after its copy
// to the device was enqueued (kept by the engine across multi-particle requests).
struct PinnedStage {
  double* pinned = nullptr;
  size_t doubles = 0;
  cudaEvent_t copied = nullptr;
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();

  int device = 0;
  cudaStream_t stream = nullptr;
  Model model;
  std::string last_error;
  long long last_samples = 0, last_launches = 0;
  long long last_not_converged = 0;

  // Run one radiation request for the current model state (single or multi particle).
  void radiation(RadRequest& rq);
  // Mixed-precision flux / spectrum of a batch of jobs in shared launches.  `out` (host) receives
  // every job's entries in job order, or with `average` the mean over the jobs (which must then
  // share observers and energies); `level_out` (host, optional) the stop levels (of the last job
  // when averaging).
  void batch(const std::vector<FieldSpec>& fields, const std::vector<BatchJob>& jobs, const double* obs,
             int64_t n_obs_total, const double* omega, int64_t n_omega_total, const osc_rad_opts& o, bool average,
             double* out, int32_t* level_out, double average_weight = 0.0);  // 0: 1 / jobs
  // The jobs' trajectories as the batched path integrates them on the device: per job 19 x n knot
  // values (t, 9 components, their 9 spline second derivatives) in job order, n in npoints.
  void batch_trajectories(const std::vector<FieldSpec>& fields, const std::vector<BatchJob>& jobs, double* out,
                          int64_t capacity, int64_t* npoints);
  // The same jobs one after another through the single-trajectory FP64 path (host RK4).
  void batch_fp64(const std::vector<FieldSpec>& fields, const std::vector<BatchJob>& jobs, const double* obs,
                  int64_t n_obs_total, const double* omega, int64_t n_omega_total, const osc_rad_opts& o,
                  bool average, double* out, int32_t* level_out);
  // Fixed-level flux and its vector-Jacobian product with respect to the half-period factors of the
  // (single) undulator that has them: grad_params = (dF/ds)^T grad_flux.  Host buffers; FP64.
  void flux_vjp(const double* obs, int64_t n_obs, const std::vector<double>& omega, int level,
                const osc_rad_opts& o, bool current_abs, const double* grad_flux, double* flux_out,
                double* grad_params, int64_t n_params, double* grad_knots = nullptr);
  // Gradient of <knot_grad, knots> (knot_grad: host, 9 x n in the knot layout x y z bx by bz ax ay az)
  // with respect to the half-period factors: reverse mode through the RK4 steps.
  void trajectory_vjp(const double* knot_grad, double* grad_params, int64_t n_params);
  // Power density on STL facets (tri: host n x 12 = vertices A, B, C and stored normal; centers:
  // host n x 3), src/OSCARSSR.cc:3154-3521; `out` / `level_out` (host) per facet.
  void power_density_stl(const double* tri, const double* centers, int64_t n, const osc_rad_opts& o, double* out,
                         int32_t* level_out);
  bool use_graphs = true;            // replay the batched front of a known shape as a CUDA graph
  // particles (this process's share) from which a mixed multi-particle request runs as one batch
  // with device trajectories instead of host trajectories and per-particle sums
  int beam_batch_min = 1024;
  // spline kernel of the batched trajectories: 0 by the chunk's shape, 1 serial sweeps, 2 block-parallel
  int spline_kernel = 0;
  long long graph_launches() const { return graph_launches_; }

  // profiling of the sample-integration kernels
  bool profiling = false;
  double prof_ms = 0;
  long long prof_launches = 0, prof_samples = 0;
  void drop_level_cache() { lev_filled_ = -1; mrec_filled_ = -1; bdmax_valid_ = false; levels_dropped_ = true; }
  double measure_fma_peak(int kind);
  // Wait for the last request's statistics; throws the errors kernels reported on the device.
  void collect();

 private:
  // trajectory on device
  DevBuf knots_;
  uint64_t knots_version_ = ~0ull;
  int64_t nknots_ = 0;
  double tstart_ = 0, tstop_ = 0;
  // level cache
  DevBuf lev_;
  int64_t lev_cap_ = 0;
  int lev_filled_ = -1;
  // levels above these in lev_ / mrec_ are the reference's extended levels (their own time spacing)
  int lev_ext_ = kMaxLevelMemory, mrec_ext_ = kMaxLevelMemory;
  void set_level_grid(int ext_from);
  DevBuf bd_bits_;                 // 32 x u64
  std::vector<double> bdmax_;      // per level, host copy
  bool bdmax_valid_ = false;
  bool levels_dropped_ = false;
  std::vector<cudaEvent_t> ev_pool_;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pending_;
  std::pair<cudaEvent_t, cudaEvent_t> timed_begin(cudaStream_t st);
  void timed_end(std::pair<cudaEvent_t, cudaEvent_t> e, cudaStream_t st);
  void collect_timings();
  // asynchronous statistics: per particle, a one-thread kernel stores the counters and the sticky
  // error word into a slot of mapped pinned memory (kStatWords words: not converged, samples, error
  // word), one event per slot
  static constexpr int kStageDoubles = 4096;
  static constexpr int kStatWords = 4;
  unsigned long long* stats_host_ = nullptr;
  double* stage_host_ = nullptr;
  // Device counter block cnt_ (16 words): [0], [1] survivor-list counts, [4..9] three 64-bit counters
  // (not converged, samples, unit counter of the running wave), [12] highest finished level -- all
  // zeroed by one memset of words 0..12 per request -- and [kCntErr] the sticky error word.
  static constexpr int kCntErr = 15;
  // pinned words the host reads back: [0] sequence word, [1] active count and [2] highest finished
  // level between waves (report_counts), [4..7] the batch statistics (two 64-bit counters), [8] the
  // batch error word, [9] the STL active count
  unsigned* ctl_host_ = nullptr;  // mapped (cudaHostAllocMapped): also written by k_report_counts
  unsigned report_seq_ = 0;
  void report_counts(const unsigned* a, const unsigned* b, unsigned* va, unsigned* vb, cudaStream_t st);
  // its sequence number; with `slot`, the kernel also stores the request's statistics there (c64[0..1]
  // and the error word)
  unsigned report_launch(const unsigned* a, const unsigned* b, cudaStream_t st, const unsigned long long* c64 = nullptr,
                         unsigned long long* slot = nullptr);
  void report_wait(unsigned seq, unsigned* va, unsigned* vb, cudaStream_t st);
  static constexpr int kStatSlots = 64;
  cudaEvent_t stats_ev_[kStatSlots] = {};
  cudaEvent_t stage_ev_ = nullptr;
  int stats_slot_ = 0;
  std::vector<int> pending_;
  // kernel variants: kind 0 = FP64 flux, 1 = FP64 power density, 2 = mixed flux, 3 = batched mixed,
  // 4 = mixed power density
  int wave_grid_[5][16] = {};
  int wave_grid(int kind, int variant);
  std::map<std::tuple<int, int, int, int>, int> tuned_;   // (kind, log2 entries, first level, last level) -> variant
  // (kind, entries, energies, last level, precision) -> highest level the last such request needed
  std::map<std::tuple<int, int64_t, int64_t, int, double>, int> prefill_hist_;
  int current_variant_[5] = {2, 0, 0, 3, 0};
  int pick_variant(int kind, RadRequest& rq, int64_t n_items, int Lfirst, int lstop, double* d_out, int32_t* d_lvl,
                   cudaStream_t st);
  bool tuning_ = false;
  // request scratch
  DevBuf obs_, nrm_, omega_, out_, lvl_, state_, part_, act_[2], cnt_;
  DevBuf fused_;                   // fused waves: rotating counts, unit counters, per-tile counters
  DevBuf acc_, acc_comp_;          // multi-particle compensated accumulation
  // mixed-precision pair records (kMixedRecordBytesPerSample per sample, level-cache indexing)
  DevBuf mrec_;
  DevBuf mrec_bd_;                 // 32 x u64: per-level beta-difference maxima of the filled records
  int64_t mrec_cap_ = 0;
  int mrec_filled_ = -1;
  uint64_t mrec_version_ = ~0ull;
  MixedFrame frame_{};
  void ensure_mixed(int L);
  void reserve_mixed(int L);
  void fill_mixed(int64_t s_begin, int64_t s_end, cudaStream_t s, bool zero_bd = true);
  void compute_frame();
 public:
  int forced_variant[5] = {-1, -1, -1, -1, -1};  // >= 0: use this compiled variant, -1: autotune per shape
  bool autotune = true;
  int variant_in_use(int kind) const { return forced_variant[kind] >= 0 ? forced_variant[kind] : current_variant_[kind]; }
  std::map<std::tuple<int, int, int, int>, int> tuned() const { return tuned_; }
 private:

  // batched path
  DevBuf b_fields_, b_fvals_, b_obs_, b_omega_, b_acc_, b_jobs_, b_knots_, b_work_, b_rec_, b_rec_ext_, b_state_, b_out_,
      b_lvl_, b_act_[2], b_part_, b_plan_, b_cnt_;
  DevBuf adj_, adj_s_, adj_r_;      // adjoint scratch
  // forward sums S (6 per entry) and flux of the last osc_flux_vjp, kept for a following call with
  // the same key (trajectory version, observers, energies, level, arithmetic, normalisation)
  DevBuf adj_sums_;
  uint64_t adj_key_ = 0;
  bool adj_key_valid_ = false;
  cudaGraphExec_t graph_exec_ = nullptr;
  long long graph_launches_ = 0;
  std::map<std::tuple<int, int64_t, int, int>, int> tuned_batch_;  // (jobs, entries, first, prefill level)
  int batch_resident(int variant);
  int tune_batch(int nj, int Lfirst, int64_t target, const DevJob* d_jobs, const BatchPlan& plan, unsigned* misc,
                 unsigned long long* m64, int64_t rec_stride);
  void radiation_beam_mixed(RadRequest& rq, int64_t N);
  double* rk4_adjoint(const double* d_kb, int param_field, int64_t n_params, cudaStream_t st);
  // RK4 adjoint states recomputed from checkpoints on the side stream (adj_z_), per trajectory version
  DevBuf adj_z_;
  uint64_t zs_version_ = ~0ull;
  bool zs_pending_ = false;
  cudaEvent_t zs_fork_ev_ = nullptr, zs_ev_ = nullptr;
  void prepare_rk4_states(cudaStream_t st);
  void join_rk4_states(cudaStream_t st);

  // stream of the running request (caches and scratch are written on it), and the ordering of
  // requests that arrive on different streams
  cudaStream_t cur_ = nullptr;
  cudaStream_t last_stream_ = nullptr;
  bool last_stream_valid_ = false;
  cudaEvent_t order_ev_ = nullptr;
  void use_stream(cudaStream_t s);
  // model.knots to the device (pinned: the same knots laid out t | y | ypp | diag in pinned memory)
  void upload_trajectory(const double* pinned = nullptr);
  void ensure_levels(int L);
  void reserve_levels(int L);
  void fill_levels(int64_t s_begin, int64_t s_end, cudaStream_t s);
  // bd_zeroed: the request prologue has zeroed the beta-step words of the levels to fill
  void prefill(bool mixed, int Lhead, int Lpre, bool bd_zeroed = false);
  void join_prefill();
  std::vector<PinnedStage> pin_pool_;  // trajectory staging of multi-particle requests
  // STL request buffers: facet geometry (A, B - A, C - A), centres, normals, per-facet state and flags
  DevBuf stl_geo_, stl_cen_, stl_nrm_, stl_state_, stl_flags_;
  // side stream of the prefill (levels above the first wave's) and its fork / join events
  cudaStream_t aux_ = nullptr;
  cudaEvent_t fork_ev_ = nullptr, join_ev_ = nullptr;
  bool join_pending_ = false;
  // Host-side inputs (observers, normals, frequencies) go up on copy_, followed by the request's
  // counter resets, while the request stream fills the level samples; the first wave waits for
  // in_ev_ (wait_inputs).
  cudaStream_t copy_ = nullptr;
  cudaEvent_t in_fork_ev_ = nullptr, in_ev_ = nullptr;
  bool inputs_pending_ = false;
  // observers / normals the waves read: the caller's device buffers, or their uploads
  const double* req_obs_ = nullptr;
  const double* req_nrm_ = nullptr;
  // frequencies staged in mapped page-locked memory (stage_host_) for the request prologue to copy
  int64_t omega_staged_ = 0;
  void wait_inputs(cudaStream_t st);
  // Result downloads of a single-particle request with host outputs, enqueued by run_single right
  // behind its statistics -- ahead of the host's last poll, so the copies need no extra round trip.
  struct ResultTail {
    bool active = false, emitted = false;
    const double* d_out = nullptr;
    const int32_t* d_lvl = nullptr;
    double* h_out = nullptr;
    int32_t* h_lvl = nullptr;
    int64_t n = 0;
  } tail_;
  int claim_stat_slot();
  void finish_request(int slot, cudaStream_t st);
  void run_single(const RadRequest& rq, int64_t n_items, double weight, double* d_out, int32_t* d_lvl,
                  cudaStream_t st);
  void check(cudaError_t e, const char* what);
};

}  // namespace osc
