// kernels_stl.cu -- power density on the facets of STL meshes (src/OSCARSSR.cc:3318-3521, the
// reference's Mode 2): for each facet i, the level samples whose ray to the facet centre crosses any
// other facet j (TTriangle3D::RayIntersectionDistance, src/TTriangle3D.cc, Moller-Trumbore) are
// skipped; the others add the power-density integrand with |N1 . normal|, and the beta-difference
// stop criterion runs over the visible samples only (src/OSCARSSR.cc:3446-3451).
//
// One CTA per facet and level.  The CTA's threads take the level's samples in chunks of kStlThreads
// (sample order = thread order inside a chunk), test each against the other facets staged in shared
// memory tiles, and find each visible sample's predecessor among the visible ones (warp ballot, then
// the previous warps' last visible samples, then the previous chunks') for the beta differences.
// Sums are reduced in a fixed order; the stop rule (src/OSCARSSR.cc:3483-3497) is applied by thread
// 0 on the facet's running state.  All FP64 operations are round-to-nearest intrinsics in the
// reference's association order, so the shadowing decisions and the beta differences are the
// reference's exactly; the sums differ only in summation order.
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"

namespace osc {
namespace dev {

constexpr int kStlThreads = 128;
constexpr int kStlTile = 128;  // facets staged in shared memory per pass (9 doubles each)

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
__device__ __forceinline__ double dot3(D3 a, D3 b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {  // TVector3D::Cross
  return {__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(b.y, a.z)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(b.z, a.x)),
          __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(b.x, a.y))};
}
__device__ __forceinline__ double mag3(D3 a) { return __dsqrt_rn(dot3(a, a)); }
__device__ __forceinline__ D3 unit3v(D3 a) {  // TVector3D::UnitVector: componentwise division by Mag()
  const double m = mag3(a);
  return {__ddiv_rn(a.x, m), __ddiv_rn(a.y, m), __ddiv_rn(a.z, m)};
}
__device__ __forceinline__ D3 orthogonal3(D3 a) {  // include/TVector3D.h:132-142
  const double xx = fabs(a.x), yy = fabs(a.y), zz = fabs(a.z);
  if (xx < yy) return xx < zz ? d3(0, a.z, -a.y) : d3(a.y, -a.x, 0);
  return yy < zz ? d3(-a.z, 0, a.x) : d3(a.y, -a.x, 0);
}

// TTriangle3D::RayIntersectionDistance for a facet given as its vertex A and edges B - A, C - A
// (f[0..8]); `dir` is the ray direction as passed (normalised again here, as the reference does).
__device__ __forceinline__ double ray_distance(const double* f, D3 origin, D3 dir_in) {
  const D3 dir = unit3v(dir_in);
  const D3 A = d3(f[0], f[1], f[2]), e1 = d3(f[3], f[4], f[5]), e2 = d3(f[6], f[7], f[8]);
  const D3 pvec = cross3(dir, e2);
  const double det = dot3(e1, pvec);
  if (det > -1e-12 && det < 1e-12) return -1;
  const double inv_det = __drcp_rn(det);
  const D3 tvec = sub3(origin, A);
  const double u = __dmul_rn(dot3(tvec, pvec), inv_det);
  if (u < 0.0 || u > 1.0) return -1;
  const D3 qvec = cross3(tvec, e1);
  const double v = __dmul_rn(dot3(dir, qvec), inv_det);
  if (v < 0.0 || __dadd_rn(u, v) > 1.0) return -1;
  const double t = __dmul_rn(dot3(e2, qvec), inv_det);
  if (t < 0) return -1;
  return t;
}

__global__ void __launch_bounds__(kStlThreads) k_stl_level(StlLevelArgs a) {
  const int64_t i = blockIdx.x;
  if (a.done[i]) return;  // uniform over the CTA
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kWarps = kStlThreads / 32;
  __shared__ double fac[kStlTile][9];
  __shared__ double wlastB[kWarps][3];
  __shared__ int wlast[kWarps];
  __shared__ double carry[3];  // beta of the level's last visible sample so far (Last_Beta)
  __shared__ double rsum[kStlThreads], rmax[kStlThreads];
  const int L = a.level;
  const int64_t ns = (int64_t)1 << L;
  const double* lev = a.lev;
  const int64_t cap = a.cap;
  const D3 obs = d3(a.centers[3 * i], a.centers[3 * i + 1], a.centers[3 * i + 2]);
  const D3 normal = d3(a.normals[3 * i], a.normals[3 * i + 1], a.normals[3 * i + 2]);
  if (tid == 0) carry[0] = carry[1] = carry[2] = 0.0;
  double psum = 0.0, bdmax = -1.0;
  for (int64_t base = 0; base < ns; base += kStlThreads) {
    const int64_t it = base + tid;  // index of the sample inside the level
    const bool active = it < ns;
    const int64_t s = ns + (active ? it : 0);
    const D3 X = d3(lev[cap + s], lev[2 * cap + s], lev[3 * cap + s]);
    const D3 B = d3(lev[4 * cap + s], lev[5 * cap + s], lev[6 * cap + s]);
    const D3 to = sub3(obs, X);
    const D3 dir = unit3v(to);
    const double dist = mag3(to);
    bool blocked = false;
    for (int64_t j0 = 0; j0 < a.n; j0 += kStlTile) {
      const int nt = (int)min((int64_t)kStlTile, a.n - j0);
      __syncthreads();
      for (int k = tid; k < nt * 9; k += kStlThreads) fac[k / 9][k % 9] = a.geometry[9 * j0 + k];
      __syncthreads();
      if (active && !blocked)
        for (int k = 0; k < nt; ++k) {
          if (j0 + k == i) continue;
          const double d = ray_distance(fac[k], X, dir);
          if (d > 0 && d < dist) {
            blocked = true;
            break;
          }
        }
    }
    const bool visible = active && !blocked;
    // predecessor of each visible sample among the visible ones (Last_Beta of the reference)
    const unsigned m = __ballot_sync(0xffffffffu, visible);
    const unsigned below = m & ((1u << lane) - 1u);
    const int src = below ? 31 - __clz(below) : lane;
    const double pbx = __shfl_sync(0xffffffffu, B.x, src), pby = __shfl_sync(0xffffffffu, B.y, src),
                 pbz = __shfl_sync(0xffffffffu, B.z, src);
    if (lane == 0) wlast[warp] = m ? 31 - __clz(m) : -1;
    if (m && lane == 31 - __clz(m)) {
      wlastB[warp][0] = B.x;
      wlastB[warp][1] = B.y;
      wlastB[warp][2] = B.z;
    }
    __syncthreads();
    if (visible) {
      D3 prev;
      if (below) {
        prev = d3(pbx, pby, pbz);
      } else {
        int w = warp - 1;
        while (w >= 0 && wlast[w] < 0) --w;
        prev = w >= 0 ? d3(wlastB[w][0], wlastB[w][1], wlastB[w][2]) : d3(carry[0], carry[1], carry[2]);
      }
      const double bd = mag3(sub3(B, prev));
      if (it > 0 && bd > bdmax) bdmax = bd;
      const D3 A = d3(lev[7 * cap + s], lev[8 * cap + s], lev[9 * cap + s]);
      const D3 N1 = unit3v(to);
      const D3 N2 = unit3v(orthogonal3(N1));
      const D3 N3 = unit3v(cross3(N1, N2));
      const double n1dn = fabs(dot3(N1, normal));
      const D3 num = cross3(N1, cross3(sub3(N1, B), A));
      const double den = pow(__dsub_rn(1.0, dot3(B, N1)), 5.0);
      const double m2 = dot3(to, to);
      const double d2 = dot3(num, N2), d3v = dot3(num, N3);
      psum = __dadd_rn(psum, __dmul_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(d2, d2), den), m2), n1dn));
      psum = __dadd_rn(psum, __dmul_rn(__ddiv_rn(__ddiv_rn(__dmul_rn(d3v, d3v), den), m2), n1dn));
    }
    __syncthreads();
    if (tid == 0) {  // the chunk's last visible sample becomes the carry
      int w = kWarps - 1;
      while (w >= 0 && wlast[w] < 0) --w;
      if (w >= 0) {
        carry[0] = wlastB[w][0];
        carry[1] = wlastB[w][1];
        carry[2] = wlastB[w][2];
      }
    }
  }
  rsum[tid] = psum;
  rmax[tid] = bdmax;
  __syncthreads();
  for (int o = kStlThreads / 2; o > 0; o >>= 1) {
    if (tid < o) {
      rsum[tid] = __dadd_rn(rsum[tid], rsum[tid + o]);
      rmax[tid] = fmax(rmax[tid], rmax[tid + o]);
    }
    __syncthreads();
  }
  if (tid != 0) return;
  // src/OSCARSSR.cc:3483-3500 on the facet's running state
  double* S = a.state + 4 * i;  // [0] sum, [1] last level value, [2] result precision, [3] last level
  const double sum = __dadd_rn(S[0], rsum[0]);
  const double ts = __dmul_rn(sum, a.dt_level);
  const double last = S[1];
  double prec = fabs(__dsub_rn(ts, last)) / last;
  const double bdm = rmax[0];
  bool done = false;
  if ((L > 8 && prec < a.precision && bdm < a.two_over_gamma) || (L > 8 && bdm < a.two_over_gamma && ts == last)) {
    done = true;
  } else if (L > 8 && ts == last) {
    done = true;
    prec = 0;
  }
  S[0] = sum;
  S[2] = prec;
  S[3] = (double)L;
  if (done) {
    a.done[i] = 1;
    a.level_out[i] = L;
  } else {
    S[1] = ts;
    atomicAdd(a.n_active, 1u);
  }
}

}  // namespace dev

cudaError_t launch_stl_level(const StlLevelArgs& a, cudaStream_t st) {
  if (a.n <= 0) return cudaSuccess;
  dev::k_stl_level<<<(unsigned)a.n, dev::kStlThreads, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace osc
