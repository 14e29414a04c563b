/*
 * oscars_oracle.c -- CPU restatement of the OSCARS radiation path (PARITY CHECKER ONLY).
 *
 * TEST INFRASTRUCTURE: loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
 * never by the oscars_b200 product.  Parity of this file with the reference is pinned by
 * tests/test_oracle_pin.py against the reference's own CPU build and the golden fixtures.
 *
 * Built with -ffp-contract=off so that every multiply and add rounds separately, exactly as the
 * reference's x86-64 build does; the association order of every expression below follows the
 * reference expression it restates (cited as file:line relative to the OSCARS source tree).
 */
#define _GNU_SOURCE
#include "oscars_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------------------------
 * Constants: include/TOSCARS.h:20-76 (the older CODATA values are kept on purpose).
 * ------------------------------------------------------------------------------------------- */
#define K_PI 3.14159265358979323846
#define K_C 2.99792458e8
#define K_H 6.62606876e-34
#define K_HBAR 1.054571596e-34
#define K_QE 1.602176462e-19
#define K_ME 9.10938356e-31
#define K_EPS0 8.854187817E-12
#define K_MU0 1.2566370614E-6
#define K_SQRT2PI 2.5066282746310002416123552393401

static double twopi(void) { return 2.0 * K_PI; }
static double fourpi(void) { return 4.0 * K_PI; }
static double kg_to_gev(double m) { return 1e-9 * m * K_C * K_C / K_QE; }       /* TOSCARS.h:75 */
static double gev_to_kg(double m) { return K_QE * m / (1e-9 * K_C * K_C); }     /* TOSCARS.h:76 */
static double ev_to_omega(double e) { return e * K_QE / K_HBAR; }               /* TOSCARS.h:70 */

#define MAX_LEVEL_MEMORY 26 /* TParticleA.h:71 */

/* ---------------------------------------------------------------------------------------------
 * 3-vectors (src/TVector3D.cc): every operator is componentwise with true division.
 * ------------------------------------------------------------------------------------------- */
typedef struct { double x, y, z; } v3;
static v3 V(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vmul(v3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
static v3 vdiv(v3 a, double s) { return V(a.x / s, a.y / s, a.z / s); }
static v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
static double vmag2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }          /* :119-123 */
static double vmag(v3 a) { return sqrt(vmag2(a)); }
static double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }     /* Dot */
static v3 vcross(v3 a, v3 b) {                                                   /* Cross */
  return V(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static v3 vunit(v3 a) { return vdiv(a, vmag(a)); }                              /* UnitVector */
static v3 vorthogonal(v3 a) {                                                    /* TVector3D.h:132-142 */
  double xx = a.x < 0.0 ? -a.x : a.x, yy = a.y < 0.0 ? -a.y : a.y, zz = a.z < 0.0 ? -a.z : a.z;
  if (xx < yy) return xx < zz ? V(0, a.z, -a.y) : V(a.y, -a.x, 0);
  return yy < zz ? V(-a.z, 0, a.x) : V(a.y, -a.x, 0);
}
/* RotateSelf(A, axis): Rodrigues matrix as written in TVector3D.cc RotateSelf. */
static v3 vrotate(v3 o, double A, v3 axis_in) {
  v3 a = vunit(axis_in);
  double ca = cos(A), sa = sin(A);
  double v0 = a.x, v1 = a.y, v2 = a.z;
  double m00 = ca + v0 * v0 * (1 - ca), m01 = v0 * v1 * (1 - ca) - v2 * sa, m02 = v0 * v2 * (1 - ca) + v1 * sa;
  double m10 = v1 * v0 * (1 - ca) + v2 * sa, m11 = ca + v1 * v1 * (1 - ca), m12 = v1 * v2 * (1 - ca) - v0 * sa;
  double m20 = v2 * v0 * (1 - ca) - v1 * sa, m21 = v2 * v1 * (1 - ca) + v0 * sa, m22 = ca + v2 * v2 * (1 - ca);
  return V(m00 * o.x + m01 * o.y + m02 * o.z, m10 * o.x + m11 * o.y + m12 * o.z,
           m20 * o.x + m21 * o.y + m22 * o.z);
}

/* Complex 3-vectors (src/TVector3DC.cc, include/TVector3DC.h) as explicit re/im pairs. */
typedef struct { double re, im; } cx;
typedef struct { cx x, y, z; } c3;
static cx cmul(cx a, cx b) { cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static cx cadd(cx a, cx b) { cx r = {a.re + b.re, a.im + b.im}; return r; }
static cx cscale(cx a, double s) { cx r = {a.re * s, a.im * s}; return r; }
static cx cconj(cx a) { cx r = {a.re, -a.im}; return r; }
static cx cdot(c3 a, c3 b) { return cadd(cadd(cmul(a.x, b.x), cmul(a.y, b.y)), cmul(a.z, b.z)); }
static c3 c3scale(c3 a, double s) { c3 r = {cscale(a.x, s), cscale(a.y, s), cscale(a.z, s)}; return r; }
static c3 c3cscale(c3 a, cx s) { c3 r = {cmul(a.x, s), cmul(a.y, s), cmul(a.z, s)}; return r; }
static c3 c3conj(c3 a) { c3 r = {cconj(a.x), cconj(a.y), cconj(a.z)}; return r; }
static double c3mag2(c3 a) { return cdot(a, c3conj(a)).re; }
/* (E . P) * P, TVector3DC::Dot without conjugation (src/OSCARSSR.cc:2000,4228) */
static c3 c3project(c3 e, c3 p) { return c3cscale(p, cdot(e, p)); }

/* ---------------------------------------------------------------------------------------------
 * Random numbers: src/TRandomA.cc uses std::mt19937 with std::normal_distribution<double> and
 * std::uniform_real_distribution<double>.  Restated from the published algorithms:
 *   MT19937 (Matsumoto & Nishimura 1998) with the C++ standard's seeding recurrence,
 *   generate_canonical<double,53> (two 32-bit draws, [C++ rand.util.canonical]),
 *   Marsaglia's polar method caching the second variate (libstdc++ normal_distribution).
 * ------------------------------------------------------------------------------------------- */
typedef struct { uint32_t mt[624]; int idx; int saved_available; double saved; } orc_rng;

static void rng_seed(orc_rng* r, uint32_t seed) {
  r->mt[0] = seed;
  for (int i = 1; i < 624; ++i)
    r->mt[i] = (uint32_t)(1812433253u * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (uint32_t)i);
  r->idx = 624;
  r->saved_available = 0;
  r->saved = 0;
}
static uint32_t rng_next(orc_rng* r) {
  if (r->idx >= 624) {
    for (int i = 0; i < 624; ++i) {
      uint32_t y = (r->mt[i] & 0x80000000u) | (r->mt[(i + 1) % 624] & 0x7fffffffu);
      r->mt[i] = r->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    r->idx = 0;
  }
  uint32_t y = r->mt[r->idx++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}
static double rng_canonical(orc_rng* r) {
  double sum = 0.0, tmp = 1.0;
  for (int k = 0; k < 2; ++k) {
    sum += (double)rng_next(r) * tmp;
    tmp *= 4294967296.0;
  }
  double ret = sum / tmp;
  if (ret >= 1.0) ret = nextafter(1.0, 0.0);
  return ret;
}
static double rng_normal(orc_rng* r) {
  if (r->saved_available) { r->saved_available = 0; return r->saved * 1.0 + 0.0; }
  double x, y, r2;
  do {
    x = 2.0 * rng_canonical(r) - 1.0;
    y = 2.0 * rng_canonical(r) - 1.0;
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0.0);
  double mult = sqrt(-2 * log(r2) / r2);
  r->saved = x * mult;
  r->saved_available = 1;
  return y * mult * 1.0 + 0.0;
}

/* ---------------------------------------------------------------------------------------------
 * Fields: ideal undulator (src/TField3D_IdealUndulator.cc:113-152) and EPU
 * (src/TField3D_IdealEPU.cc:116-170), summed by TFieldContainer::GetF (src/TFieldContainer.cc:85-104)
 * ------------------------------------------------------------------------------------------- */
typedef struct {
  int kind; /* 0 undulator, 1 EPU, 2 grid */
  v3 field, field_b, period, center;
  int nperiods;
  double phase, taper, frequency, frequency_phase, time_offset;
  double period_length, und_length;
  v3 period_unit;
  double* half_scale; /* undulator: per half-period factors of the full-strength region, or NULL */
  int n_half;
  /* grid (TField3D_Grid): n, start, step, stop per axis, dimension code, values (3 per point) */
  long gn[3];
  double gstart[3], gstep[3], gstop[3];
  int gdim;
  double* gval;
  v3 grot;
} orc_field;

enum { GD_X = 0, GD_Y, GD_Z, GD_XY, GD_XZ, GD_YZ, GD_XYZ };

/* TVector3D::RotateSelfXYZ: about x, then y, then z. */
static v3 vrotxyz(v3 v, v3 r) {
  double s = sin(r.x), c = cos(r.x), t = v.y;
  v.y = c * t - s * v.z;
  v.z = s * t + c * v.z;
  s = sin(r.y); c = cos(r.y); t = v.z;
  v.z = c * t - s * v.x;
  v.x = s * t + c * v.x;
  s = sin(r.z); c = cos(r.z); t = v.x;
  v.x = c * t - s * v.y;
  v.y = s * t + c * v.y;
  return v;
}

/* One sinusoidal block with the 1/4 and 3/4 end poles, as in IdealUndulator::GetF. */
static v3 und_block(const orc_field* f, v3 amp, double d, double phase_shift, double taper_corr) {
  double L = f->und_length, lam = f->period_length;
  v3 F = V(0, 0, 0);
  if (d > L / 2. + phase_shift || d < -L / 2. + phase_shift) return F;
  double s = sin(twopi() * (d - phase_shift) / lam);
  if (d < -L / 2. + phase_shift + lam || d > L / 2. + phase_shift - lam) {
    if (d < -L / 2. + phase_shift + lam / 2. || d > L / 2. + phase_shift - lam / 2.)
      F = vmul(vmul(vmul(amp, 0.25), s), taper_corr);
    else
      F = vmul(vmul(vmul(amp, 0.75), s), taper_corr);
  } else {
    F = vmul(vmul(amp, s), taper_corr);
    if (f->half_scale) { /* half-period k of the full-strength region, counted from its start */
      long k = (long)((d - (-L / 2. + phase_shift + lam)) / (lam / 2.));
      k = k < 0 ? 0 : (k >= f->n_half ? f->n_half - 1 : k);
      F = vmul(F, f->half_scale[k]);
    }
  }
  return F;
}

/* Grid field, src/TField3D_Grid.cc:153-283. */
static v3 gval(const orc_field* f, long i) { return V(f->gval[3 * i], f->gval[3 * i + 1], f->gval[3 * i + 2]); }
static v3 glerp(v3 a, v3 b, double d, double step) { return vadd(a, vdiv(vmul(vsub(b, a), d), step)); }

static v3 grid_eval(const orc_field* f, v3 XIN, double T) {
  v3 X = vsub(vrotxyz(XIN, f->grot), f->center);
  double p[3] = {X.x, X.y, X.z};
  long ni[3] = {0, 0, 0};
  double di[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a) {
    if (f->gn[a] > 1 && (p[a] <= f->gstart[a] || p[a] >= f->gstop[a])) return V(0, 0, 0);
  }
  for (int a = 0; a < 3; ++a) {
    if (f->gn[a] > 1) {
      ni[a] = (long)((p[a] - f->gstart[a]) / f->gstep[a]);
      di[a] = (p[a] - f->gstart[a]) - ni[a] * f->gstep[a];
      if (ni[a] > f->gn[a] - 2) ni[a] = f->gn[a] - 2;
    }
  }
  long NY = f->gn[1], NZ = f->gn[2];
#define GI(ix, iy, iz) ((ix) * NY * NZ + (iy) * NZ + (iz))
  long nx = ni[0], ny = ni[1], nz = ni[2];
  double dx = di[0], dy = di[1], dz = di[2];
  v3 F;
  switch (f->gdim) {
    case GD_XYZ: {
      v3 v00 = glerp(gval(f, GI(nx, ny, nz)), gval(f, GI(nx + 1, ny, nz)), dx, f->gstep[0]);
      v3 v10 = glerp(gval(f, GI(nx, ny + 1, nz)), gval(f, GI(nx + 1, ny + 1, nz)), dx, f->gstep[0]);
      v3 v01 = glerp(gval(f, GI(nx, ny, nz + 1)), gval(f, GI(nx + 1, ny, nz + 1)), dx, f->gstep[0]);
      v3 v11 = glerp(gval(f, GI(nx, ny + 1, nz + 1)), gval(f, GI(nx + 1, ny + 1, nz + 1)), dx, f->gstep[0]);
      v3 v0 = glerp(v00, v10, dy, f->gstep[1]);
      v3 v1 = glerp(v01, v11, dy, f->gstep[1]);
      F = glerp(v0, v1, dz, f->gstep[2]);
      break;
    }
    case GD_X: F = glerp(gval(f, nx), gval(f, nx + 1), dx, f->gstep[0]); break;
    case GD_Y: F = glerp(gval(f, ny), gval(f, ny + 1), dy, f->gstep[1]); break;
    case GD_Z: F = glerp(gval(f, nz), gval(f, nz + 1), dz, f->gstep[2]); break;
    case GD_XY: {
      v3 v0 = glerp(gval(f, GI(nx, ny, 0)), gval(f, GI(nx + 1, ny, 0)), dx, f->gstep[0]);
      v3 v1 = glerp(gval(f, GI(nx, ny + 1, 0)), gval(f, GI(nx + 1, ny + 1, 0)), dx, f->gstep[0]);
      F = glerp(v0, v1, dy, f->gstep[1]);
      break;
    }
    case GD_XZ: {
      v3 v0 = glerp(gval(f, GI(nx, 0, nz)), gval(f, GI(nx + 1, 0, nz)), dx, f->gstep[0]);
      v3 v1 = glerp(gval(f, GI(nx, 0, nz + 1)), gval(f, GI(nx + 1, 0, nz + 1)), dx, f->gstep[0]);
      F = glerp(v0, v1, dz, f->gstep[2]);
      break;
    }
    default: {
      v3 v0 = glerp(gval(f, GI(0, ny, nz)), gval(f, GI(0, ny + 1, nz)), dy, f->gstep[1]);
      v3 v1 = glerp(gval(f, GI(0, ny, nz + 1)), gval(f, GI(0, ny + 1, nz + 1)), dy, f->gstep[1]);
      F = glerp(v0, v1, dz, f->gstep[2]);
      break;
    }
  }
#undef GI
  return vmul(F, cos(twopi() * f->frequency * (T + f->time_offset) + f->frequency_phase));
}

static v3 field_eval(const orc_field* f, v3 X, double T) {
  if (f->kind == 2) return grid_eval(f, X, T);
  double d = vdot(vsub(X, f->center), f->period_unit);
  double taper_corr = 1 + d * f->taper;
  v3 F;
  if (f->kind == 0) {
    double ps = f->phase * vmag(f->period) / twopi();
    F = und_block(f, f->field, d, ps, taper_corr);
  } else {
    /* EPU: two blocks with phase shifts +/- phase/2 (TField3D_IdealEPU.cc:127-165) */
    double ps = f->phase / 2. * vmag(f->period) / twopi();
    F = und_block(f, f->field, d, ps, taper_corr);
    ps = -f->phase / 2. * vmag(f->period) / twopi();
    F = vadd(F, und_block(f, f->field_b, d, ps, taper_corr));
  }
  if (f->frequency == 0) return F;
  return vmul(F, cos(twopi() * f->frequency * (T + f->time_offset) + f->frequency_phase));
}

/* ---------------------------------------------------------------------------------------------
 * Simulation state
 * ------------------------------------------------------------------------------------------- */
typedef struct {
  double q, m, gamma, qomg, current;
  v3 x0, b0;
  double t0;
  int set;
} orc_particle;

typedef struct {
  int type_set;
  double q, m, current, e0, t0;
  v3 x0, u0, b0, hdir, vdir;
  double sigma_e;
  double emit[2], eta[2];
  double tw_beta[2], tw_alpha[2], tw_gamma[2];
  double tw_beta_x0[2], tw_alpha_x0[2], tw_gamma_x0[2];
  v3 lattice_ref;
  int distribution;
} orc_beam;

typedef struct {
  long n;
  double* t;     /* n */
  double* y;     /* 9 x n : x y z bx by bz ax ay az */
  double* ypp;   /* 9 x n */
  double tstart, tstop;
  double* level[MAX_LEVEL_MEMORY + 1]; /* cached 10 x 2^L SoA */
} orc_traj;

struct orc_sim {
  orc_field fields[64];
  int nfields;
  orc_beam beams[16];   /* TParticleBeamContainer: beams and the running sums of their weights */
  double wsum[16];
  int nbeams;
  int has_beam;
  orc_particle p;
  double ctstart, ctstop;
  long npoints, npoints_per_meter;
  orc_rng rng;
  orc_traj tr;
  int error_gamma;
  int traj_method;        /* 0 RK4, 1 RKAS (OSCARSSR::SetTrajectoryCalculation) */
  double traj_precision;  /* RKAS precision, default 1e-6 (src/OSCARSSR.cc:47) */
  char err[256];
};

static int fail(orc_sim* s, int code, const char* msg) {
  snprintf(s->err, sizeof s->err, "%s", msg);
  return code;
}

static void traj_clear(orc_traj* tr) {
  free(tr->t); free(tr->y); free(tr->ypp);
  tr->t = tr->y = tr->ypp = NULL;
  for (int l = 0; l <= MAX_LEVEL_MEMORY; ++l) { free(tr->level[l]); tr->level[l] = NULL; }
  tr->n = 0;
}

orc_sim* orc_new(void) {
  orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
  if (!s) return NULL;
  s->npoints_per_meter = 10000; /* OSCARSSR.cc:42 */
  s->traj_precision = 1e-6;     /* OSCARSSR.cc:47 */
  rng_seed(&s->rng, 5489u);
  return s;
}
static void fields_free(orc_sim* s) {
  for (int i = 0; i < s->nfields; ++i) {
    free(s->fields[i].half_scale);
    free(s->fields[i].gval);
    s->fields[i].half_scale = NULL;
    s->fields[i].gval = NULL;
  }
  s->nfields = 0;
}
void orc_free(orc_sim* s) {
  if (!s) return;
  traj_clear(&s->tr);
  fields_free(s);
  free(s);
}
const char* orc_last_error(const orc_sim* s) { return s->err; }

int orc_clear_fields(orc_sim* s) { fields_free(s); traj_clear(&s->tr); return ORC_OK; }

static int add_field(orc_sim* s, int kind, const double* fa, const double* fb, const double* period,
                     int nperiods, const double* center, double phase, double taper, double freq,
                     double fphase, double toff) {
  if (s->nfields >= 64) return fail(s, ORC_ERR_RANGE, "too many fields");
  orc_field* f = &s->fields[s->nfields++];
  memset(f, 0, sizeof *f);
  f->kind = kind;
  f->field = V(fa[0], fa[1], fa[2]);
  if (fb) f->field_b = V(fb[0], fb[1], fb[2]);
  f->period = V(period[0], period[1], period[2]);
  f->nperiods = nperiods;
  f->center = V(center[0], center[1], center[2]);
  f->phase = phase; f->taper = taper; f->frequency = freq;
  f->frequency_phase = fphase; f->time_offset = toff;
  f->period_length = vmag(f->period);                       /* Init :94-98 */
  f->period_unit = vunit(f->period);
  f->und_length = vmag(f->period) * (nperiods + 2);
  traj_clear(&s->tr);                                        /* OSCARSSR.cc:157-169 */
  return ORC_OK;
}
int orc_add_undulator(orc_sim* s, const double field[3], const double period[3], int nperiods,
                      const double center[3], double phase, double taper, double frequency,
                      double frequency_phase, double time_offset) {
  return add_field(s, 0, field, NULL, period, nperiods, center, phase, taper, frequency,
                   frequency_phase, time_offset);
}
int orc_add_epu(orc_sim* s, const double field_a[3], const double field_b[3], const double period[3],
                int nperiods, const double center[3], double phase, double taper, double frequency,
                double frequency_phase, double time_offset) {
  return add_field(s, 1, field_a, field_b, period, nperiods, center, phase, taper, frequency,
                   frequency_phase, time_offset);
}

int orc_set_half_period_scale(orc_sim* s, const double* scale, int n) {
  if (s->nfields < 1 || s->fields[s->nfields - 1].kind != 0) return fail(s, ORC_ERR_STATE, "last field is not an undulator");
  orc_field* f = &s->fields[s->nfields - 1];
  if (n != 2 * f->nperiods) return fail(s, ORC_ERR_RANGE, "n_half_periods must be 2 * nperiods");
  free(f->half_scale);
  f->half_scale = (double*)malloc(sizeof(double) * n);
  if (!f->half_scale) return fail(s, ORC_ERR_ALLOC, "allocation failed");
  memcpy(f->half_scale, scale, sizeof(double) * n);
  f->n_half = n;
  traj_clear(&s->tr);
  return ORC_OK;
}

int orc_add_grid(orc_sim* s, const long n[3], const double start[3], const double step[3], const double stop[3],
                 const double* values, const double rotations[3], const double translation[3], double frequency,
                 double frequency_phase, double time_offset) {
  if (s->nfields >= 64) return fail(s, ORC_ERR_RANGE, "too many fields");
  int hx = n[0] > 1, hy = n[1] > 1, hz = n[2] > 1;
  int dim = hx && hy && hz ? GD_XYZ : hx && hy ? GD_XY : hx && hz ? GD_XZ : hy && hz ? GD_YZ : hx ? GD_X : hy ? GD_Y
          : hz ? GD_Z : -1;
  if (dim < 0) return fail(s, ORC_ERR_RANGE, "invalid dimensions");
  long N = n[0] * n[1] * n[2];
  orc_field* f = &s->fields[s->nfields];
  memset(f, 0, sizeof *f);
  f->gval = (double*)malloc(sizeof(double) * 3 * N);
  if (!f->gval) return fail(s, ORC_ERR_ALLOC, "allocation failed");
  memcpy(f->gval, values, sizeof(double) * 3 * N);
  ++s->nfields;
  f->kind = 2;
  for (int a = 0; a < 3; ++a) {
    f->gn[a] = n[a]; f->gstart[a] = start[a]; f->gstep[a] = step[a]; f->gstop[a] = stop[a];
  }
  f->gdim = dim;
  f->grot = V(rotations[0], rotations[1], rotations[2]);
  f->center = V(translation[0], translation[1], translation[2]);
  f->frequency = frequency; f->frequency_phase = frequency_phase; f->time_offset = time_offset;
  traj_clear(&s->tr);
  return ORC_OK;
}

static v3 field_sum(const orc_sim* s, v3 X, double T) {
  v3 sum = V(0, 0, 0);
  for (int i = 0; i < s->nfields; ++i) sum = vadd(sum, field_eval(&s->fields[i], X, T));
  return sum;
}
int orc_get_bfield(const orc_sim* s, const double x[3], double t, double out[3]) {
  v3 b = field_sum(s, V(x[0], x[1], x[2]), t);
  out[0] = b.x; out[1] = b.y; out[2] = b.z;
  return ORC_OK;
}

/* ---------------------------------------------------------------------------------------------
 * Particle and beam: src/TParticleA.cc:400-483, src/TParticleBeam.cc, src/OSCARSSR_Python.cc
 * add_particle_beam :3699-4100 / set_particle_beam :3561-3576.
 * ------------------------------------------------------------------------------------------- */
static void particle_set_conditions(orc_particle* p, v3 x0, v3 b0, double t0) {
  p->x0 = x0; p->b0 = b0; p->t0 = t0;
  double beta2 = vmag2(b0) > 0 ? vmag2(b0) : 0;                        /* SetGamma :444-459 */
  if (beta2 != 1) {
    p->gamma = beta2 != 0 ? 1.0 / sqrt(1.0 - beta2) : 1;
    if (!(p->m == 0 || p->gamma == 0)) p->qomg = p->q / p->m / p->gamma; /* :464-472 */
  }
  p->set = 1;
}

static void beam_twiss_at_x0(orc_beam* b) {                            /* TParticleBeam.cc:262-277 */
  v3 dx = vsub(b->x0, b->lattice_ref);
  double D = vmag(dx);
  double L = vdot(dx, b->u0) >= 0 ? D : -1. * D;
  for (int i = 0; i < 2; ++i) {
    b->tw_beta_x0[i] = b->tw_beta[i] - 2 * L * b->tw_alpha[i] + L * L * b->tw_gamma[i];
    b->tw_alpha_x0[i] = b->tw_alpha[i] - L * b->tw_gamma[i];
    b->tw_gamma_x0[i] = b->tw_gamma[i];
  }
}

static int type_qm(int code, double charge, double mass, double* q, double* m) {
  switch (code) {                                                      /* TParticleA.cc:78-121 */
    case 0: *q = -K_QE; *m = K_ME; return 0;
    case 1: *q = K_QE; *m = K_ME; return 0;
    case 2: *q = -K_QE; *m = gev_to_kg(0.1056583715); return 0;
    case 3: *q = K_QE; *m = gev_to_kg(0.1056583715); return 0;
    case 4: *q = K_QE; *m = gev_to_kg(0.938272046); return 0;
    case 5: *q = -K_QE; *m = gev_to_kg(0.938272046); return 0;
    case 6: *q = K_QE; *m = gev_to_kg(0.13957018); return 0;
    case 7: *q = -K_QE; *m = gev_to_kg(0.13957018); return 0;
    case 8: *q = charge; *m = mass; return 0;
    default: return -1;
  }
}

int orc_set_ctstartstop(orc_sim* s, double start, double stop) {       /* OSCARSSR.cc:637-647 */
  s->npoints = (long)(s->npoints_per_meter * (stop - start));
  s->ctstart = start;
  s->ctstop = stop;
  return ORC_OK;
}
int orc_set_npoints_trajectory(orc_sim* s, long n) { s->npoints = n; return ORC_OK; }
long orc_get_npoints_trajectory(const orc_sim* s) { return s->npoints; }
int orc_set_seed(orc_sim* s, int seed) { rng_seed(&s->rng, (uint32_t)seed); return ORC_OK; }
double orc_uniform(orc_sim* s) { return rng_canonical(&s->rng); }
double orc_normal(orc_sim* s) { return rng_normal(&s->rng); }

/* TParticleBeam::GetNewParticle("ideal") (TParticleBeam.cc:667-688) */
static void beam_ideal_particle(const orc_beam* b, orc_particle* p) {
  double g = b->e0 / kg_to_gev(b->m) < 1 ? 1 : b->e0 / kg_to_gev(b->m);
  double beta = g != 1 ? sqrt(1.0 - 1.0 / (g * g)) : 0;
  p->q = b->q; p->m = b->m; p->current = b->current;
  particle_set_conditions(p, b->x0, vmul(b->u0, beta), b->t0);
}

/* TParticleBeamContainer::GetRandomBeamIndexByWeight (TParticleBeamContainer.cc:135-166) */
static int pick_beam(orc_sim* s) {
  if (s->nbeams == 1) return 0;
  double r = rng_canonical(&s->rng) * s->wsum[s->nbeams - 1];
  for (int i = 0; i != s->nbeams; ++i)
    if (r < s->wsum[i]) return i;
  return s->nbeams - 1;
}

/* TParticleBeam::GetNewParticle() Gaussian branch (TParticleBeam.cc:713-774) */
static void beam_random_particle(orc_sim* s, const orc_beam* b, orc_particle* p) {
  if (b->distribution == ORC_DIST_FILAMENT || b->distribution == ORC_DIST_NONE) {
    beam_ideal_particle(b, p);
    return;
  }
  double PI = K_PI;
  p->q = b->q; p->m = b->m; p->current = b->current;
  double mgev = kg_to_gev(b->m);
  double enew = b->e0 + b->sigma_e * rng_normal(&s->rng);
  if (enew < mgev) enew = mgev;
  double ge = enew / mgev < 1 ? 1 : enew / mgev;
  double beta = ge != 1 ? sqrt(1.0 - 1.0 / (ge * ge)) : 0;
  double de = (enew - b->e0) / b->e0;
  v3 xn = b->x0;
  v3 bn = vmul(vcross(b->hdir, b->vdir), beta);
  if (b->distribution == ORC_DIST_GAUSSIAN) {
    if (b->emit[0] * b->emit[0] + b->emit[1] * b->emit[1] > 1e-99) {
      int hc = b->tw_alpha_x0[0] > 0 ? -1 : 1;
      int vc = b->tw_alpha_x0[1] > 0 ? -1 : 1;
      double hsx = sqrt(b->emit[0] * b->tw_beta_x0[0]);
      double hsxp = sqrt(b->emit[0] * b->tw_gamma_x0[0]);
      double hr0 = b->emit[0] / (hsx * hsxp);
      double hrho = sqrt(1 - hr0 * hr0);
      double vsx = sqrt(b->emit[1] * b->tw_beta_x0[1]);
      double vsxp = sqrt(b->emit[1] * b->tw_gamma_x0[1]);
      double vr0 = b->emit[1] / (vsx * vsxp);
      double vrho = sqrt(1 - vr0 * vr0);
      double hu = rng_canonical(&s->rng);
      double hv = rng_canonical(&s->rng);
      double hX = hsx * sqrt(-2 * log(hu)) * (sqrt(1 - hrho * hrho) * cos(2 * PI * hv) + hrho * sin(2 * PI * hv));
      double hXP = hc * hsxp * sqrt(-2 * log(hu)) * sin(2 * PI * hv);
      double vu = rng_canonical(&s->rng);
      double vv = rng_canonical(&s->rng);
      double vX = vsx * sqrt(-2 * log(vu)) * (sqrt(1 - vrho * vrho) * cos(2 * PI * vv) + vrho * sin(2 * PI * vv));
      double vXP = vc * vsxp * sqrt(-2 * log(vu)) * sin(2 * PI * vv);
      /* `XNew += H * hX + eta * dE/E` adds the scalar to every component (implicit TVector3D(double)) */
      double eh = b->eta[0] * de, ev = b->eta[1] * de;
      v3 th = vmul(b->hdir, hX);
      xn = vadd(xn, V(th.x + eh, th.y + eh, th.z + eh));
      v3 tv = vmul(b->vdir, vX);
      xn = vadd(xn, V(tv.x + ev, tv.y + ev, tv.z + ev));
      bn = vrotate(bn, hXP, b->vdir);
      bn = vrotate(bn, vXP, vneg(b->hdir));
    }
  } else { /* KV branch (TParticleBeam.cc:776-848) */
    int hc = b->tw_alpha_x0[0] > 0 ? -1 : 1;
    int vc = b->tw_alpha_x0[1] > 0 ? -1 : 1;
    double hTheta = rng_canonical(&s->rng) * 2 * PI;
    double vTheta = rng_canonical(&s->rng) * 2 * PI;
    double hAX = sqrt(b->emit[0] * b->tw_beta_x0[0]) * cos(hTheta);
    double vAX = sqrt(b->emit[1] * b->tw_beta_x0[1]) * cos(vTheta);
    double hAXP = -sqrt(b->emit[0] / b->tw_beta_x0[0]) * (b->tw_alpha_x0[0] * cos(hTheta) + sin(hTheta));
    double vAXP = -sqrt(b->emit[1] / b->tw_beta_x0[1]) * (b->tw_alpha_x0[1] * cos(vTheta) + sin(vTheta));
    double hR = sqrt(hAX * hAX + hAXP * hAXP);
    double vR = sqrt(vAX * vAX + vAXP * vAXP);
    double hRT = atan(hAXP / hAX), vRT = atan(vAXP / vAX);
    if (hAX < 0 && hAXP > 0) hRT += PI; else if (hAX < 0 && hAXP < 0) hRT -= PI;
    if (vAX < 0 && vAXP > 0) vRT += PI; else if (vAX < 0 && vAXP < 0) vRT -= PI;
    double hNR = sqrt(rng_canonical(&s->rng)) * hR;
    double vNR = sqrt(rng_canonical(&s->rng)) * vR;
    double hX = hNR * cos(hRT), vX = vNR * cos(vRT);
    double hXP = hNR * sin(hRT) * hc, vXP = vNR * sin(vRT) * vc;
    xn = vadd(xn, vmul(b->hdir, hX));
    xn = vadd(xn, vmul(b->vdir, vX));
    bn = vmul(vcross(b->hdir, b->vdir), beta);
    bn = vrotate(bn, hXP, b->vdir);
    bn = vrotate(bn, vXP, vneg(b->hdir));
  }
  particle_set_conditions(p, xn, bn, b->t0);
}

/* add_particle_beam (OSCARSSR_Python.cc:3796-4096) with TParticleBeam's constructor, its setters and
 * SetPredefinedBeam (TParticleBeam.cc:97-125, 135-206, 219-350, 374-381, 551-612); x0 / d0 already
 * rotated and translated, `horizontal` the given direction or -d0.Orthogonal() of the unrotated one.
 * append = 0 replaces the beams (set_particle_beam). */
int orc_set_beam(orc_sim* s, int type_code, double charge, double mass, double energy_GeV,
                 const double x0[3], const double d0[3], double t0, double current,
                 const double horizontal[3], int has_horizontal, double sigma_energy_GeV,
                 const double emittance[2], int has_emittance, const double beta[2],
                 const double alpha[2], int has_beta, int has_alpha, const double eta[2],
                 int distribution_override, const double ctstartstop[2], int has_ctstartstop,
                 const double gamma[2], int has_gamma, const double lattice_ref[3], int has_lattice_ref,
                 int predefined, int has_d0, double weight, int append) {
  if (!append) s->nbeams = 0;
  if (s->nbeams >= 16) return fail(s, ORC_ERR_ARG, "too many beams");
  int first = s->nbeams == 0;
  orc_beam bb;
  orc_beam* b = &bb;
  memset(b, 0, sizeof *b);
  if (predefined) {                                                     /* SetPredefinedBeam */
    if (type_qm(0, 0, 0, &b->q, &b->m)) return fail(s, ORC_ERR_ARG, "bad particle type");
    b->current = 0.500;
    b->e0 = 3 < kg_to_gev(b->m) ? b->m : 3;
    b->u0 = vunit(V(0, 0, 1));
    b->t0 = 0;
    b->x0 = V(0, 0, 0);
    beam_twiss_at_x0(b);
    b->emit[0] = 0.55e-9; b->emit[1] = 0.008e-9;
    b->lattice_ref = V(0, 0, 0);
    beam_twiss_at_x0(b);
    double bt0 = predefined == 2 ? 18 : 1.5, bt1 = predefined == 2 ? 3.1 : 0.8;
    b->tw_beta[0] = bt0; b->tw_beta[1] = bt1;
    b->tw_gamma[0] = (1. + 0. * 0.) / bt0; b->tw_gamma[1] = (1. + 0. * 0.) / bt1;
    b->tw_alpha[0] = 0; b->tw_alpha[1] = 0;
    beam_twiss_at_x0(b);
    b->sigma_e = predefined == 1 ? 0 : 3. * 0.00089;
    b->vdir = vunit(V(0, 1, 0));                                        /* SetVerticalDirection */
    b->hdir = vunit(vcross(b->vdir, b->u0));
    b->distribution = predefined == 1 ? ORC_DIST_FILAMENT : ORC_DIST_GAUSSIAN;
    if (energy_GeV >= 0) b->e0 = energy_GeV < kg_to_gev(b->m) ? b->m : energy_GeV;
  }
  if (energy_GeV == -1) energy_GeV = 0;
  if (energy_GeV < 0) return fail(s, ORC_ERR_ARG, "negative energy");
  if (weight == 0) weight = 1;
  if (weight <= 0) return fail(s, ORC_ERR_ARG, "Particle weight cannot be negative");
  v3 dir = d0 ? V(d0[0], d0[1], d0[2]) : V(0, 0, 1);
  v3 pos = x0 ? V(x0[0], x0[1], x0[2]) : V(0, 0, 0);
  v3 hd = has_horizontal ? V(horizontal[0], horizontal[1], horizontal[2]) : vneg(vorthogonal(dir));
  hd = vunit(hd);
  if (!predefined) {                           /* TParticleBeam 10-argument constructor (TParticleBeam.cc:97-125) */
    if (type_qm(type_code, charge, mass, &b->q, &b->m)) return fail(s, ORC_ERR_ARG, "bad particle type");
    b->x0 = pos;
    b->u0 = vmag2(dir) > 0 ? vunit(dir) : V(0, 0, 0);
    b->e0 = energy_GeV < kg_to_gev(b->m) ? b->m : energy_GeV;
    b->t0 = t0;
    b->current = current != 0 ? current : b->q;                       /* TParticleA::SetCurrent */
  } else {
    if (has_d0) b->u0 = vunit(dir);                                    /* SetU0 */
    b->x0 = pos;                                                       /* SetX0 */
    beam_twiss_at_x0(b);
  }
  {
    double g = b->e0 / kg_to_gev(b->m);
    double bt = sqrt(1.0 - 1.0 / (g * g));
    b->b0 = vmul(b->u0, bt);
  }
  /* SetHorizontalDirection (TParticleBeam.cc:374-381) */
  b->hdir = vunit(hd);
  b->vdir = vneg(vunit(vcross(hd, b->u0)));
  if (has_emittance) {
    b->emit[0] = emittance[0]; b->emit[1] = emittance[1];
    b->distribution = ORC_DIST_GAUSSIAN;
  } else if (!predefined) {
    b->distribution = ORC_DIST_FILAMENT;
  }
  if (distribution_override >= 0) b->distribution = distribution_override;
  if (sigma_energy_GeV < 0) return fail(s, ORC_ERR_ARG, "'sigma_energy_GeV' cannot be less than zero");
  if (sigma_energy_GeV > 0) b->sigma_e = sigma_energy_GeV;
  v3 ref = has_lattice_ref ? V(lattice_ref[0], lattice_ref[1], lattice_ref[2]) : V(0, 0, 0);
  b->lattice_ref = ref;                                                 /* SetTwissLatticeReference */
  beam_twiss_at_x0(b);
  int bag = (has_beta ? 4 : 0) | (has_alpha ? 2 : 0) | (has_gamma ? 1 : 0);
  if (bag == 7) {                                                       /* SetTwissParameters */
    for (int i = 0; i < 2; ++i) { b->tw_beta[i] = beta[i]; b->tw_alpha[i] = alpha[i]; b->tw_gamma[i] = gamma[i]; }
  } else if (bag == 6 || bag == 4) {                                    /* SetTwissBetaAlpha */
    double a0 = bag == 6 ? alpha[0] : 0, a1 = bag == 6 ? alpha[1] : 0;
    if (beta[0] <= 0 || beta[1] <= 0) return fail(s, ORC_ERR_ARG, "Beta cannot be <= 0");
    b->tw_beta[0] = beta[0]; b->tw_beta[1] = beta[1];
    b->tw_gamma[0] = (1. + a0 * a0) / beta[0];
    b->tw_gamma[1] = (1. + a1 * a1) / beta[1];
    b->tw_alpha[0] = a0; b->tw_alpha[1] = a1;
  } else if (bag == 5) {                                                /* SetTwissBetaGamma */
    for (int i = 0; i < 2; ++i) {
      b->tw_beta[i] = beta[i]; b->tw_alpha[i] = sqrt(gamma[i] * beta[i] - 1); b->tw_gamma[i] = gamma[i];
    }
  } else if (bag == 3) {                                                /* SetTwissAlphaGamma */
    if (gamma[0] == 0 || gamma[1] == 0) return fail(s, ORC_ERR_ARG, "Gamma cannot be <= 0");
    for (int i = 0; i < 2; ++i) {
      b->tw_beta[i] = (1. + alpha[i] * alpha[i]) / gamma[i]; b->tw_alpha[i] = alpha[i]; b->tw_gamma[i] = gamma[i];
    }
  }
  if (bag == 7 || bag == 6 || bag == 5 || bag == 4 || bag == 3) {
    if (has_lattice_ref) b->lattice_ref = ref;
    beam_twiss_at_x0(b);
  }
  if (eta) { b->eta[0] = eta[0]; b->eta[1] = eta[1]; }
  if (t0 != 0) b->t0 = t0;
  s->beams[s->nbeams] = *b;
  s->wsum[s->nbeams] = s->nbeams == 0 ? weight : s->wsum[s->nbeams - 1] + weight;
  s->nbeams++;
  s->has_beam = 1;
  if (has_ctstartstop) orc_set_ctstartstop(s, ctstartstop[0], ctstartstop[1]);
  else orc_set_ctstartstop(s, -3, 3);                                    /* Python.cc:4087-4093 */
  if (first) beam_ideal_particle(&s->beams[0], &s->p);                  /* SetNewParticle("", "ideal") */
  traj_clear(&s->tr);
  return ORC_OK;
}

/* OSCARSSR::SetNewParticle(beam, ideal or random) (OSCARSSR.cc:510-524); beam < 0 picks one by weight. */
int orc_set_new_particle_of(orc_sim* s, int beam, int ideal) {
  if (!s->has_beam) return fail(s, ORC_ERR_STATE, "no beam defined");
  if (beam >= s->nbeams) return fail(s, ORC_ERR_RANGE, "beam name not in map");
  const orc_beam* b = &s->beams[beam < 0 ? pick_beam(s) : beam];
  if (ideal) beam_ideal_particle(b, &s->p);
  else beam_random_particle(s, b, &s->p);
  traj_clear(&s->tr);
  return ORC_OK;
}

int orc_set_new_particle(orc_sim* s, int ideal) { return orc_set_new_particle_of(s, -1, ideal); }

int orc_set_particle(orc_sim* s, const double x0[3], const double b0[3], double t0) {
  if (!s->has_beam) return fail(s, ORC_ERR_STATE, "no beam defined");
  orc_particle p;
  memset(&p, 0, sizeof p);
  p.q = s->beams[0].q; p.m = s->beams[0].m; p.current = s->beams[0].current;
  particle_set_conditions(&p, V(x0[0], x0[1], x0[2]), V(b0[0], b0[1], b0[2]), t0);
  s->p = p;
  traj_clear(&s->tr);
  return ORC_OK;
}

int orc_get_particle(const orc_sim* s, double x0[3], double b0[3], double* t0, double* gamma,
                     double* q, double* m, double* current) {
  x0[0] = s->p.x0.x; x0[1] = s->p.x0.y; x0[2] = s->p.x0.z;
  b0[0] = s->p.b0.x; b0[1] = s->p.b0.y; b0[2] = s->p.b0.z;
  *t0 = s->p.t0; *gamma = s->p.gamma; *q = s->p.q; *m = s->p.m; *current = s->p.current;
  return ORC_OK;
}

/* ---------------------------------------------------------------------------------------------
 * RK4 trajectory: OSCARSSR::CalculateTrajectoryRK4 (src/OSCARSSR.cc:910-1009), DerivativesB
 * (:1247-1279) and RK4 with gamma-error step halving (:1321-1386).
 * ------------------------------------------------------------------------------------------- */
static void derivs(orc_sim* s, double t, const double x[6], double dxdt[6]) {
  double one_minus = (1. - (x[1] * x[1] + x[3] * x[3] + x[5] * x[5]) / (K_C * K_C));
  if (one_minus <= 0) { s->error_gamma = 1; return; }
  v3 B = field_sum(s, V(x[0], x[2], x[4]), t);
  double k = s->p.qomg;
  dxdt[0] = x[1];
  dxdt[1] = k * (-x[5] * B.y + x[3] * B.z);
  dxdt[2] = x[3];
  dxdt[3] = k * (x[5] * B.x - x[1] * B.z);
  dxdt[4] = x[5];
  dxdt[5] = k * (x[1] * B.y - x[3] * B.x);
}

static void rk4(orc_sim* s, double y[6], double dydx[6], double x, double h, double yout[6]) {
  double dym[6], dyt[6], yt[6], ytest[6];
  double hh = h * 0.5, h6 = h / 6.0, xh = x + hh;
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dydx[i];
  derivs(s, xh, yt, dyt);
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dyt[i];
  derivs(s, xh, yt, dym);
  for (int i = 0; i < 6; ++i) { yt[i] = y[i] + h * dym[i]; dym[i] += dyt[i]; }
  derivs(s, x + h, yt, dyt);
  for (int i = 0; i < 6; ++i) ytest[i] = y[i] + h6 * (dydx[i] + dyt[i] + 2.0 * dym[i]);
  int this_err = 1. - (ytest[1] * ytest[1] + ytest[3] * ytest[3] + ytest[5] * ytest[5]) / (K_C * K_C) <= 0;
  if (s->error_gamma || this_err) {
    s->error_gamma = 0;
    double yhalf[6];
    derivs(s, x, y, dydx);
    rk4(s, y, dydx, x, h / 2., yhalf);
    derivs(s, x + h / 2., yhalf, dydx);
    rk4(s, yhalf, dydx, x + h / 2., h / 2., ytest);
  }
  for (int i = 0; i < 6; ++i) yout[i] = ytest[i];
}

typedef struct { double* v; long n, cap; } dbuf; /* 10 doubles per point (t, x, b, a/c) */
static int dbuf_push(dbuf* d, const double* x, const double* dxdt, double t) {
  if (d->n == d->cap) {
    long nc = d->cap ? d->cap * 2 : 1024;
    double* nv = (double*)realloc(d->v, sizeof(double) * 10 * nc);
    if (!nv) return -1;
    d->v = nv; d->cap = nc;
  }
  double* r = d->v + 10 * d->n++;
  r[0] = t; r[1] = x[0]; r[2] = x[2]; r[3] = x[4];
  r[4] = x[1] / K_C; r[5] = x[3] / K_C; r[6] = x[5] / K_C;
  r[7] = dxdt[1] / K_C; r[8] = dxdt[3] / K_C; r[9] = dxdt[5] / K_C;
  return 0;
}
static void dbuf_reverse(dbuf* d) {
  for (long i = 0, j = d->n - 1; i < j; ++i, --j)
    for (int k = 0; k < 10; ++k) { double t = d->v[10 * i + k]; d->v[10 * i + k] = d->v[10 * j + k]; d->v[10 * j + k] = t; }
}

static int spline_setup(orc_traj* tr); /* below */

/* ---- RKAS: OSCARSSR::RKCK / RKQS / PropogateRKAS (src/OSCARSSR.cc:1392-1618) ------------------- */
static void rkck(orc_sim* s, const double* x, const double* dxdt, double t, double h, double* xout, double* xerr) {
  static const double a2 = 0.2, a3 = 0.3, a4 = 0.6, a5 = 1.0, a6 = 0.875;
  static const double b21 = 0.2, b31 = 3.0 / 40.0, b32 = 9.0 / 40.0, b41 = 0.3, b42 = -0.9, b43 = 1.2;
  static const double b51 = -11.0 / 54.0, b52 = 2.5, b53 = -70.0 / 27.0, b54 = 35.0 / 27.0;
  static const double b61 = 1631.0 / 55296.0, b62 = 175.0 / 512.0, b63 = 575.0 / 13824.0;
  static const double b64 = 44275.0 / 110592.0, b65 = 253.0 / 4096.0;
  static const double c1 = 37.0 / 378.0, c3 = 250.0 / 621.0, c4 = 125.0 / 594.0, c6 = 512.0 / 1771.0;
  static const double dc5 = -277.00 / 14336.0;
  const double dc1 = c1 - 2825.0 / 27648.0, dc3 = c3 - 18575.0 / 48384.0, dc4 = c4 - 13525.0 / 55296.0;
  const double dc6 = c6 - 0.25;
  double dx2[6], dx3[6], dx4[6], dx5[6], dx6[6], xt[6];
  for (int i = 0; i != 6; ++i) xt[i] = x[i] + b21 * h * dxdt[i];
  derivs(s, t + a2 * h, xt, dx2);
  for (int i = 0; i != 6; ++i) xt[i] = x[i] + h * (b31 * dxdt[i] + b32 * dx2[i]);
  derivs(s, t + a3 * h, xt, dx3);
  for (int i = 0; i != 6; ++i) xt[i] = x[i] + h * (b41 * dxdt[i] + b42 * dx2[i] + b43 * dx3[i]);
  derivs(s, t + a4 * h, xt, dx4);
  for (int i = 0; i != 6; ++i) xt[i] = x[i] + h * (b51 * dxdt[i] + b52 * dx2[i] + b53 * dx3[i] + b54 * dx4[i]);
  derivs(s, t + a5 * h, xt, dx5);
  for (int i = 0; i != 6; ++i) xt[i] = x[i] + h * (b61 * dxdt[i] + b62 * dx2[i] + b63 * dx3[i] + b64 * dx4[i] + b65 * dx5[i]);
  derivs(s, t + a6 * h, xt, dx6);
  for (int i = 0; i != 6; ++i) xout[i] = x[i] + h * (c1 * dxdt[i] + c3 * dx3[i] + c4 * dx4[i] + c6 * dx6[i]);
  for (int i = 0; i != 6; ++i) xerr[i] = h * (dc1 * dxdt[i] + dc3 * dx3[i] + dc4 * dx4[i] + dc5 * dx5[i] + dc6 * dx6[i]);
}

static int rkqs(orc_sim* s, double* x, double* dxdt, double* t, double htry, double prec, const double* xscale,
                double delta_t, double* hnext) {
  double h = htry, max_error = 0, xt[6], xe[6];
  for (;;) {
    s->error_gamma = 0;
    rkck(s, x, dxdt, *t, h, xt, xe);
    max_error = 0.0;
    for (int i = 0; i != 6; ++i) max_error = fmax(max_error, fabs(xe[i] / xscale[i]));
    max_error /= prec;
    if (max_error <= 1.0 && !s->error_gamma) break;
    double htemp = s->error_gamma ? 0.25 * h : 0.9 * h * pow(max_error, -0.25);
    h = (h >= 0.0 ? fmax(htemp, 0.1 * h) : fmin(htemp, 0.1 * h));
    if ((*t) + h == *t) return fail(s, ORC_ERR_RANGE, "stepsize underflow in rkqs.  Possible you have a discontinuous field");
  }
  *hnext = max_error > 1.89e-4 ? 0.9 * h * pow(max_error, -0.2) : 5.0 * h;
  if (fabs(*hnext) > delta_t) *hnext = delta_t * (*hnext >= 0 ? 1 : -1);
  *t += h;
  for (int i = 0; i != 6; ++i) x[i] = xt[i];
  return ORC_OK;
}

static int propagate_rkas(orc_sim* s, double* xstart, double T1, double T2, double prec, double delta_t, dbuf* d) {
  double x[6], dxdt[6] = {0, 0, 0, 0, 0, 0}, xscale[6], hnext = 0;
  double t = T1, h = (T2 >= T1 ? delta_t : -delta_t);
  for (int i = 0; i != 6; ++i) x[i] = xstart[i];
  for (long nstp = 0; nstp != 10000000; ++nstp) {
    derivs(s, t, x, dxdt);
    for (int i = 0; i != 6; ++i) xscale[i] = fabs(x[i]) + fabs(dxdt[i] * h) + 1.0e-30;
    if (dbuf_push(d, x, dxdt, t)) return fail(s, ORC_ERR_ALLOC, "alloc");
    if ((t + h - T2) * (t + h - T1) > 0.0) h = T2 - t;
    int rc = rkqs(s, x, dxdt, &t, h, prec, xscale, delta_t, &hnext);
    if (rc) return rc;
    if ((t - T2) * (T2 - T1) >= 0.0) {
      for (int i = 0; i != 6; ++i) xstart[i] = x[i];
      if (dbuf_push(d, x, dxdt, t)) return fail(s, ORC_ERR_ALLOC, "alloc");
      return ORC_OK;
    }
    if (fabs(hnext) <= 1e-30) return fail(s, ORC_ERR_RANGE, "Reached minimum stepsize in PropogateRKAS without convergence");
    h = hnext;
  }
  return fail(s, ORC_ERR_RANGE, "Too many steps taken in routine PropogateRKAS");
}

int orc_set_trajectory_calculation(orc_sim* s, int method, double precision) {
  s->traj_method = method;
  if (precision != -1) s->traj_precision = precision;
  return ORC_OK;
}

int orc_calculate_trajectory(orc_sim* s) {
  if (!s->p.set) return fail(s, ORC_ERR_STATE, "particle not initialized.  make sure you have a particle or beam defined");
  if (s->ctstart > s->p.t0 || s->ctstop < s->p.t0)
    return fail(s, ORC_ERR_RANGE, "start time is greater than T0 or stop time is less than T0");
  if (s->ctstart >= s->ctstop)
    return fail(s, ORC_ERR_RANGE, "start time is greater than stop time.  check that set_ctstartstop is set");
  traj_clear(&s->tr);
  s->error_gamma = 0;
  double const DeltaT = ((s->ctstop - s->ctstart) / K_C / (s->npoints - 1));
  size_t nf = (size_t)(1 + (s->ctstop - s->p.t0) / K_C / DeltaT);
  size_t nb = (size_t)((s->p.t0 - s->ctstart) / K_C / DeltaT);
  double x[6], dxdt[6] = {0, 0, 0, 0, 0, 0};
  dbuf d = {0, 0, 0};
  x[0] = s->p.x0.x; x[1] = s->p.b0.x * K_C; x[2] = s->p.x0.y;
  x[3] = s->p.b0.y * K_C; x[4] = s->p.x0.z; x[5] = s->p.b0.z * K_C;
  derivs(s, s->p.t0 / K_C, x, dxdt);
  if (s->traj_method == 1) {  /* OSCARSSR::CalculateTrajectoryRKAS (src/OSCARSSR.cc:1015-1072) */
    int rc = propagate_rkas(s, x, s->p.t0 / K_C, s->ctstop / K_C, s->traj_precision, DeltaT, &d);
    if (rc) { free(d.v); return rc; }
    dbuf_reverse(&d);
    x[0] = s->p.x0.x; x[1] = s->p.b0.x * K_C; x[2] = s->p.x0.y;
    x[3] = s->p.b0.y * K_C; x[4] = s->p.x0.z; x[5] = s->p.b0.z * K_C;
    derivs(s, s->p.t0 / K_C, x, dxdt);
    rc = propagate_rkas(s, x, s->p.t0 / K_C, s->ctstart / K_C, s->traj_precision, DeltaT, &d);
    if (rc) { free(d.v); return rc; }
    nf = nb = 0;
  }
  for (size_t i = 0; i != nf; ++i) {
    double t = s->p.t0 / K_C + DeltaT * i;
    if (i == 0) derivs(s, t, x, dxdt);
    if (dbuf_push(&d, x, dxdt, t)) { free(d.v); return fail(s, ORC_ERR_ALLOC, "alloc"); }
    derivs(s, t, x, dxdt);
    rk4(s, x, dxdt, t, DeltaT, x);
  }
  if (s->traj_method != 1) dbuf_reverse(&d);
  x[0] = s->p.x0.x; x[1] = s->p.b0.x * K_C; x[2] = s->p.x0.y;
  x[3] = s->p.b0.y * K_C; x[4] = s->p.x0.z; x[5] = s->p.b0.z * K_C;
  double const dtr = -DeltaT;
  for (size_t i = 0; i != nb; ++i) {
    double t1 = s->p.t0 / K_C + dtr * (i);
    double t2 = s->p.t0 / K_C + dtr * (i + 1);
    derivs(s, t1, x, dxdt);
    rk4(s, x, dxdt, t1, dtr, x);
    if (dbuf_push(&d, x, dxdt, t2)) { free(d.v); return fail(s, ORC_ERR_ALLOC, "alloc"); }
  }
  dbuf_reverse(&d);
  if (d.n < 2) { free(d.v); return fail(s, ORC_ERR_RANGE, "Not enough points in this trajectory"); }
  orc_traj* tr = &s->tr;
  tr->n = d.n;
  tr->t = (double*)malloc(sizeof(double) * d.n);
  tr->y = (double*)malloc(sizeof(double) * 9 * d.n);
  tr->ypp = (double*)malloc(sizeof(double) * 9 * d.n);
  if (!tr->t || !tr->y || !tr->ypp) { free(d.v); traj_clear(tr); return fail(s, ORC_ERR_ALLOC, "alloc"); }
  for (long i = 0; i < d.n; ++i) {
    tr->t[i] = d.v[10 * i];
    for (int k = 0; k < 9; ++k) tr->y[k * d.n + i] = d.v[10 * i + 1 + k];
  }
  free(d.v);
  tr->tstart = tr->t[0];
  tr->tstop = tr->t[tr->n - 1];
  if (tr->n < 3) { traj_clear(tr); return fail(s, ORC_ERR_RANGE, "TSpline1D3 does not see enough points for interpolation.  Please use >= 3 points"); }
  spline_setup(tr);
  return ORC_OK;
}

long orc_trajectory_npoints(const orc_sim* s) { return s->tr.n; }
int orc_get_trajectory(const orc_sim* s, double* out, long cap) {
  long n = s->tr.n;
  if (cap < 10 * n) return ORC_ERR_RANGE;
  memcpy(out, s->tr.t, sizeof(double) * n);
  memcpy(out + n, s->tr.y, sizeof(double) * 9 * n);
  return ORC_OK;
}
int orc_get_spline_ypp(const orc_sim* s, double* out, long cap) {
  if (cap < 9 * s->tr.n) return ORC_ERR_RANGE;
  memcpy(out, s->tr.ypp, sizeof(double) * 9 * s->tr.n);
  return ORC_OK;
}

/* ---------------------------------------------------------------------------------------------
 * Clamped cubic spline: TSpline1D3::Derivatives / GetValue (include/TOMATH.h:92-203), applied to
 * every one of the 9 components (TParticleTrajectoryPoint arithmetic is componentwise).
 * ------------------------------------------------------------------------------------------- */
static int spline_setup(orc_traj* tr) {
  long N = tr->n;
  const double* X = tr->t;
  double* u = (double*)malloc(sizeof(double) * N);
  if (!u) return -1;
  for (int k = 0; k < 9; ++k) {
    const double* Y = tr->y + k * N;
    double* ypp = tr->ypp + k * N;
    double dydx0 = (Y[1] - Y[0]) / (X[1] - X[0]);
    ypp[0] = -0.5;
    u[0] = (3. / (X[1] - X[0])) * ((Y[1] - Y[0]) / (X[1] - X[0]) - dydx0);
    for (long i = 1; i < N - 1; ++i) {
      double sig = (X[i] - X[i - 1]) / (X[i + 1] - X[i - 1]);
      double p = sig * ypp[i - 1] + 2;
      ypp[i] = (sig - 1.) / p;
      u[i] = (Y[i + 1] - Y[i]) / (X[i + 1] - X[i]) - (Y[i] - Y[i - 1]) / (X[i] - X[i - 1]);
      u[i] = (6. * u[i] / (X[i + 1] - X[i - 1]) - sig * u[i - 1]) / p;
    }
    double qn = 0.5;
    double dydxN = (Y[N - 1] - Y[N - 2]) / (X[N - 1] - X[N - 2]);
    double un = (3. / (X[N - 1] - X[N - 2])) * (dydxN - (Y[N - 1] - Y[N - 2]) / (X[N - 1] - X[N - 2]));
    ypp[N - 1] = (un - qn * u[N - 2]) / (qn * ypp[N - 2] + 1.);
    for (long j = N - 2; j >= 0; --j) ypp[j] = ypp[j] * ypp[j + 1] + u[j];
  }
  free(u);
  return 0;
}

static void spline_eval(const orc_traj* tr, double x, double out[9]) {
  long klo = 0, khi = tr->n - 1, k;
  const double* X = tr->t;
  while (khi - klo > 1) {
    k = (khi + klo) >> 1;
    if (X[k] > x) khi = k; else klo = k;
  }
  double h = X[khi] - X[klo];
  double a = (X[khi] - x) / h;
  double b = (x - X[klo]) / h;
  for (int c = 0; c < 9; ++c) {
    const double* Y = tr->y + c * tr->n;
    const double* P = tr->ypp + c * tr->n;
    out[c] = a * Y[klo] + b * Y[khi] + ((a * a * a - a) * P[klo] + (b * b * b - b) * P[khi]) * (h * h) / 6.;
  }
}

/* Level L samples: t = tS + T/2^(L+1) + i*T/2^L, i < 2^L (TParticleTrajectoryInterpolated.cc:124-158);
 * extended levels use spacing T/(2^L - 1) (TParticleTrajectoryInterpolatedPoints.cc:36-61). */
static void level_time(const orc_traj* tr, int L, int extended, double* tstart, double* spacing) {
  *tstart = tr->tstart + (tr->tstop - tr->tstart) / pow(2., L + 1);
  *spacing = extended ? (tr->tstop - tr->tstart) / (pow(2., L) - 1)
                      : (tr->tstop - tr->tstart) / pow(2., L);
}

static const double* get_level(orc_traj* tr, int L) {
  if (tr->level[L]) return tr->level[L];
  long np = (long)pow(2, L);
  double* v = (double*)malloc(sizeof(double) * 10 * np);
  if (!v) return NULL;
  double ts, sp, r[9];
  level_time(tr, L, 0, &ts, &sp);
  for (long i = 0; i < np; ++i) {
    double T = ts + sp * (double)i;
    spline_eval(tr, T, r);
    v[i] = T;
    for (int c = 0; c < 9; ++c) v[(1 + c) * np + i] = r[c];
  }
  tr->level[L] = v;
  return v;
}

int orc_get_level(orc_sim* s, int level, double* out, long cap) {
  if (level < 0 || level > MAX_LEVEL_MEMORY) return ORC_ERR_RANGE;
  long np = (long)pow(2, level);
  if (cap < 10 * np) return ORC_ERR_RANGE;
  const double* v = get_level(&s->tr, level);
  if (!v) return ORC_ERR_ALLOC;
  memcpy(out, v, sizeof(double) * 10 * np);
  return ORC_OK;
}

static double delta_t_inclusive(const orc_traj* tr, int L) {          /* :224-237 */
  return (tr->tstop - tr->tstart) / (pow(2., L + 1) - 1);
}

/* Sample iT of level L (memory or extended), as 10 doubles. */
typedef struct { const double* mem; long np; double ts, sp; int ext; } level_view;
static int level_open(orc_traj* tr, int L, int lstop_mem, level_view* lv) {
  if (L <= lstop_mem) {
    lv->mem = get_level(tr, L);
    if (!lv->mem) return -1;
    lv->np = (long)pow(2, L);
    lv->ext = 0;
  } else {
    lv->mem = NULL;
    lv->np = (long)(int)pow(2, L);
    level_time(tr, L, 1, &lv->ts, &lv->sp);
    lv->ext = 1;
  }
  return 0;
}
static void level_point(const orc_traj* tr, const level_view* lv, long i, double* T, v3* X, v3* B, v3* A) {
  double r[9];
  if (!lv->ext) {
    long n = lv->np;
    *T = lv->mem[i];
    for (int c = 0; c < 9; ++c) r[c] = lv->mem[(1 + c) * n + i];
  } else {
    *T = lv->ts + lv->sp * (double)i;
    spline_eval(tr, *T, r);
  }
  *X = V(r[0], r[1], r[2]); *B = V(r[3], r[4], r[5]); *A = V(r[6], r[7], r[8]);
}

/* ---------------------------------------------------------------------------------------------
 * Polarization vector (src/OSCARSSR.cc:4116-4150)
 * ------------------------------------------------------------------------------------------- */
static c3 c3real(v3 a) { c3 r = {{a.x, 0}, {a.y, 0}, {a.z, 0}}; return r; }
static c3 pol_vector(int pol, double angle, v3 hor, v3 prop) {
  v3 vert = vunit(vcross(prop, hor));
  double k = 1. / sqrt(2);
  c3 r = {{0, 0}, {0, 0}, {0, 0}};
  switch (pol) {
    case ORC_POL_LH: return c3real(hor);
    case ORC_POL_LV: return c3real(vert);
    case ORC_POL_LINEAR: return c3real(vrotate(hor, angle, prop));
    case ORC_POL_CL: {
      /* 1/sqrt(2) * (H + V*i): V*i = (v*0, v*1) */
      c3 p = {{hor.x + vert.x * 0, 0 + vert.x * 1}, {hor.y + vert.y * 0, 0 + vert.y * 1}, {hor.z + vert.z * 0, 0 + vert.z * 1}};
      return c3scale(p, k);
    }
    case ORC_POL_CR: {
      c3 p = {{hor.x - vert.x * 0, 0 - vert.x * 1}, {hor.y - vert.y * 0, 0 - vert.y * 1}, {hor.z - vert.z * 0, 0 - vert.z * 1}};
      return c3scale(p, k);
    }
    default: return r;
  }
}

/* ---------------------------------------------------------------------------------------------
 * Frequency-domain integral for one (observer, omega) pair.  Shared by CalculateFluxPoints
 * (src/OSCARSSR.cc:4157-4268) and CalculateSpectrumPoints (:1948-2038): level ladder, integrand
 * :4202-4220, stop rule :4233-4238, final scaling :4246-4267.
 * Returns the value selected by `quantity`; *level_out receives the stop level or -1.
 * ------------------------------------------------------------------------------------------- */
typedef struct { int lstop_mem, lstop_ext; double precision; c3 pol; int project; } fd_opts;

static int fd_point(orc_traj* tr, v3 obs, double omega, const fd_opts* o, double C0, double C2,
                    double weight, int quantity, double* value, int* level_out, int* converged) {
  c3 sum = {{0, 0}, {0, 0}, {0, 0}};
  double this_mag = -1, last_mag = -1, last_phase = -1, max_dphase = 0;
  int last_level = 0, result_level = -1;
  double result_precision = -1;
  for (int L = 0; L <= o->lstop_ext; ++L) {
    last_level = L;
    level_view lv;
    if (level_open(tr, L, o->lstop_mem, &lv)) return -1;
    max_dphase = 0;
    for (long i = 0; i != lv.np; ++i) {
      double T; v3 X, B, A;
      level_point(tr, &lv, i, &T, &X, &B, &A);
      v3 R = vsub(obs, X);
      v3 N = vunit(R);
      double D = vmag(R);
      double phase = -omega * (T + D / K_C);
      double ptv = fabs(phase - last_phase);
      if (i != 0 && ptv > max_dphase) max_dphase = ptv;
      last_phase = phase;
      double cph, sph;
      sincos(phase, &sph, &cph);
      double ndb = vdot(N, B);
      double p2 = (1 - ndb) * (1 - ndb);
      v3 NB = vsub(N, B);
      v3 t1 = vdiv(vmul(NB, 1 - vmag2(B)), D * D * p2);
      v3 t2 = vdiv(vcross(N, vcross(NB, A)), D * p2);
      v3 ew = vadd(t1, t2);
      sum.x.re += ew.x * cph; sum.x.im += ew.x * sph;
      sum.y.re += ew.y * cph; sum.y.im += ew.y * sph;
      sum.z.re += ew.z * cph; sum.z.im += ew.z * sph;
    }
    c3 ts = c3scale(sum, delta_t_inclusive(tr, L));
    if (o->project) ts = c3project(ts, o->pol);
    this_mag = c3mag2(ts);
    result_precision = fabs(this_mag - last_mag) / last_mag;
    if ((L > 8 && result_precision < o->precision && max_dphase < K_PI) ||
        (L > 8 && max_dphase < K_PI && this_mag == last_mag)) {
      result_level = L;
      break;
    }
    last_mag = this_mag;
  }
  *converged = result_level != -1;
  sum = c3scale(sum, C0 * delta_t_inclusive(tr, last_level));
  if (o->project) sum = c3project(sum, o->pol);
  *level_out = result_level;
  switch (quantity) {
    case 1: *value = result_precision * weight; break;
    case 2: *value = ((double)result_level) * weight; break;
    default: *value = C2 * c3mag2(sum) * weight; break;
  }
  return 0;
}

static void fd_options(int pol, double angle, const double* hor, const double* prop, double precision,
                       int max_level, int max_level_ext, fd_opts* o) {
  o->lstop_mem = max_level >= -1 && max_level <= MAX_LEVEL_MEMORY ? max_level : MAX_LEVEL_MEMORY;
  o->lstop_ext = max_level_ext > o->lstop_mem ? max_level_ext : o->lstop_mem;
  o->precision = precision;
  o->pol = pol_vector(pol, angle, V(hor[0], hor[1], hor[2]), V(prop[0], prop[1], prop[2]));
  o->project = pol != ORC_POL_ALL && c3mag2(o->pol) > 0.001;
}

static void kahan_add(double* sum, double* comp, double v) {          /* T3DScalarContainer.cc:35-51 */
  double S = *sum, y = v - *comp, t = S + y;
  *comp = (t - S) - y;
  *sum = t;
}

static int ensure_trajectory(orc_sim* s) {
  if (!s->p.set) {
    if (!s->has_beam) return fail(s, ORC_ERR_STATE, "no beam defined");
    beam_random_particle(s, &s->beams[pick_beam(s)], &s->p);
  }
  if (s->tr.n == 0) return orc_calculate_trajectory(s);
  return ORC_OK;
}

int orc_flux(orc_sim* s, const double* obs, long n_obs, double energy_eV, int pol, double angle,
             const double horizontal[3], const double propagation[3], double precision,
             int max_level, int max_level_extended, int nparticles, int quantity, double* out,
             int* out_level) {
  fd_opts o;
  fd_options(pol, angle, horizontal, propagation, precision, max_level, max_level_extended, &o);
  double omega = ev_to_omega(energy_eV);
  double* comp = (double*)calloc((size_t)n_obs, sizeof(double));
  if (!comp) return fail(s, ORC_ERR_ALLOC, "alloc");
  for (long i = 0; i < n_obs; ++i) out[i] = 0;
  int np = nparticles > 0 ? nparticles : 1;
  double weight = nparticles > 0 ? 1.0 / (double)nparticles : 1;
  for (int ip = 0; ip < np; ++ip) {
    int rc;
    if (nparticles > 0) {
      if ((rc = orc_set_new_particle(s, 0))) { free(comp); return rc; }
      if ((rc = orc_calculate_trajectory(s))) { free(comp); return rc; }
    } else if ((rc = ensure_trajectory(s))) { free(comp); return rc; }
    double C0 = s->p.q / (fourpi() * K_C * K_EPS0 * K_SQRT2PI);                    /* :4106 */
    double C2 = fourpi() * s->p.current / (K_H * fabs(s->p.q) * K_MU0 * K_C) * 1e-6 * 0.001; /* :4109 */
    for (long i = 0; i < n_obs; ++i) {
      double v; int lvl, conv;
      if (fd_point(&s->tr, V(obs[3 * i], obs[3 * i + 1], obs[3 * i + 2]), omega, &o, C0, C2, weight,
                   quantity, &v, &lvl, &conv)) { free(comp); return fail(s, ORC_ERR_ALLOC, "alloc"); }
      kahan_add(&out[i], &comp[i], v);
      if (out_level) out_level[i] = lvl;
    }
  }
  free(comp);
  return ORC_OK;
}

int orc_spectrum(orc_sim* s, const double obs[3], const double* energies_eV, long n_e, int pol,
                 double angle, const double horizontal[3], const double propagation[3],
                 double precision, int max_level, int max_level_extended, int nparticles,
                 int quantity, double* out, int* out_level) {
  fd_opts o;
  fd_options(pol, angle, horizontal, propagation, precision, max_level, max_level_extended, &o);
  double* comp = (double*)calloc((size_t)n_e, sizeof(double));
  if (!comp) return fail(s, ORC_ERR_ALLOC, "alloc");
  for (long i = 0; i < n_e; ++i) out[i] = 0;
  int np = nparticles > 0 ? nparticles : 1;
  double weight = nparticles > 0 ? 1.0 / (double)nparticles : 1;
  for (int ip = 0; ip < np; ++ip) {
    int rc;
    if (nparticles > 0) {
      if ((rc = orc_set_new_particle(s, 0))) { free(comp); return rc; }
      if ((rc = orc_calculate_trajectory(s))) { free(comp); return rc; }
    } else if ((rc = ensure_trajectory(s))) { free(comp); return rc; }
    double C0 = s->p.q / (fourpi() * K_C * K_EPS0 * K_SQRT2PI);                           /* :1885 */
    double C2 = fourpi() * fabs(s->p.current) / (K_H * fabs(s->p.q) * K_MU0 * K_C) * 1e-6 * 0.001; /* :1888 */
    for (long i = 0; i < n_e; ++i) {
      double v; int lvl, conv;
      double omega = ev_to_omega(energies_eV[i]);                                       /* TSpectrumContainer.cc:262 */
      if (fd_point(&s->tr, V(obs[0], obs[1], obs[2]), omega, &o, C0, C2, weight, quantity, &v, &lvl, &conv)) {
        free(comp); return fail(s, ORC_ERR_ALLOC, "alloc");
      }
      kahan_add(&out[i], &comp[i], v);
      if (out_level) out_level[i] = lvl;
    }
  }
  free(comp);
  return ORC_OK;
}

/* ---------------------------------------------------------------------------------------------
 * Power density: OSCARSSR::CalculatePowerDensityPoints (src/OSCARSSR.cc:2817-2976)
 * ------------------------------------------------------------------------------------------- */
static int pd_point(orc_traj* tr, v3 obs, v3 normal, int directional, int lstop_mem, int lstop_ext,
                    double precision, double gamma, double scale, double weight, int quantity,
                    double* value, int* level_out) {
  double this_sum = -1, last_sum = -1, sum = 0, result_precision = -1;
  int last_level = 0, result_level = -1;
  (void)this_sum;
  for (int L = 0; L <= lstop_ext; ++L) {
    last_level = L;
    v3 last_beta = V(0, 0, 0);
    double bdmax = -1;
    level_view lv;
    if (level_open(tr, L, lstop_mem, &lv)) return -1;
    for (long i = 0; i != lv.np; ++i) {
      double T; v3 X, B, A;
      level_point(tr, &lv, i, &T, &X, &B, &A);
      double bd = vmag(vsub(B, last_beta));
      if (i > 0 && bd > bdmax) bdmax = bd;
      last_beta = B;
      v3 N1 = vunit(vsub(obs, X));
      v3 N2 = vunit(vorthogonal(N1));
      v3 N3 = vunit(vcross(N1, N2));
      double n1dn = vdot(N1, normal);
      if (directional && n1dn <= 0) continue;
      v3 num = vcross(N1, vcross(vsub(N1, B), A));
      double den = pow(1 - vdot(B, N1), 5);
      double m2 = vmag2(vsub(obs, X));
      double d2 = vdot(num, N2), d3 = vdot(num, N3);
      sum += d2 * d2 / den / m2 * n1dn;
      sum += d3 * d3 / den / m2 * n1dn;
    }
    double ts = sum * delta_t_inclusive(tr, L);
    result_precision = fabs(ts - last_sum) / last_sum;
    if ((L > 8 && result_precision < precision && bdmax < 2. / gamma) ||
        (L > 8 && bdmax < 2. / gamma && ts == last_sum)) {
      result_level = L;
      last_sum = ts;
      break;
    } else if (L > 8 && ts == last_sum) {
      result_level = L;
      result_precision = 0;
      break;
    }
    last_sum = ts;
  }
  sum *= scale * delta_t_inclusive(tr, last_level);
  sum /= 1e6;
  if (!directional && sum < 0) sum *= -1;
  *level_out = result_level;
  switch (quantity) {
    case 1: *value = result_precision * weight; break;
    case 2: *value = ((double)result_level) * weight; break;
    default: *value = sum * weight; break;
  }
  return 0;
}

int orc_power_density(orc_sim* s, const double* obs, const double* normals, long n_obs,
                      int directional, double precision, int max_level, int max_level_extended,
                      int nparticles, int quantity, double* out, int* out_level) {
  int lstop_mem = max_level >= -1 && max_level <= MAX_LEVEL_MEMORY ? max_level : MAX_LEVEL_MEMORY;
  int lstop_ext = max_level_extended > lstop_mem ? max_level_extended : lstop_mem;
  double* comp = (double*)calloc((size_t)n_obs, sizeof(double));
  if (!comp) return fail(s, ORC_ERR_ALLOC, "alloc");
  for (long i = 0; i < n_obs; ++i) out[i] = 0;
  int np = nparticles > 0 ? nparticles : 1;
  double weight = nparticles > 0 ? 1.0 / (double)nparticles : 1;
  for (int ip = 0; ip < np; ++ip) {
    int rc;
    if (nparticles > 0) {
      if ((rc = orc_set_new_particle(s, 0))) { free(comp); return rc; }
      if ((rc = orc_calculate_trajectory(s))) { free(comp); return rc; }
    } else if ((rc = ensure_trajectory(s))) { free(comp); return rc; }
    /* |Q I| / (16 pi^2 eps0 c) (src/OSCARSSR.cc:2945) */
    double scale = fabs(s->p.q * s->p.current) / (16 * (K_PI * K_PI) * K_EPS0 * K_C);
    for (long i = 0; i < n_obs; ++i) {
      double v; int lvl;
      if (pd_point(&s->tr, V(obs[3 * i], obs[3 * i + 1], obs[3 * i + 2]),
                   V(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]), directional, lstop_mem,
                   lstop_ext, precision, s->p.gamma, scale, weight, quantity, &v, &lvl)) {
        free(comp); return fail(s, ORC_ERR_ALLOC, "alloc");
      }
      kahan_add(&out[i], &comp[i], v);
      if (out_level) out_level[i] = lvl;
    }
  }
  free(comp);
  return ORC_OK;
}

/* ---------------------------------------------------------------------------------------------
 * Power density on STL facets: OSCARSSR::CalculatePowerDensityPointsSTL (src/OSCARSSR.cc:3318-3521,
 * the Mode 2 path: a sample is skipped when any other facet lies between it and the facet centre)
 * with TTriangle3D::RayIntersectionDistance (src/TTriangle3D.cc, Moller-Trumbore).
 * tri: n x 12 (vertices A, B, C, normal N as stored); centers: n x 3 (TTriangle3D::fCenter).
 * ------------------------------------------------------------------------------------------- */
static double ray_intersection_distance(const double* T, v3 origin, v3 dir_in) {
  v3 A = V(T[0], T[1], T[2]), B = V(T[3], T[4], T[5]), C = V(T[6], T[7], T[8]);
  v3 dir = vunit(dir_in);
  v3 edge1 = vsub(B, A), edge2 = vsub(C, A);
  v3 pvec = vcross(dir, edge2);
  double det = vdot(edge1, pvec);
  if (det > -1e-12 && det < 1e-12) return -1;
  double inv_det = 1.0 / det;
  v3 tvec = vsub(origin, A);
  double u = vdot(tvec, pvec) * inv_det;
  if (u < 0.0 || u > 1.0) return -1;
  v3 qvec = vcross(tvec, edge1);
  double v = vdot(dir, qvec) * inv_det;
  if (v < 0.0 || u + v > 1.0) return -1;
  double t = vdot(edge2, qvec) * inv_det;
  if (t < 0) return -1;
  return t;
}

int orc_power_density_stl(orc_sim* s, const double* tri, const double* centers, long n, double precision,
                          int max_level, int max_level_extended, int nparticles, int quantity, double* out,
                          int* out_level) {
  int lstop_mem = max_level >= -1 && max_level <= MAX_LEVEL_MEMORY ? max_level : MAX_LEVEL_MEMORY;
  int lstop_ext = max_level_extended > lstop_mem ? max_level_extended : lstop_mem;
  for (long i = 0; i < n; ++i) out[i] = 0;
  int np = nparticles > 0 ? nparticles : 1;
  double weight = nparticles > 0 ? 1.0 / (double)nparticles : 1;
  for (int ip = 0; ip < np; ++ip) {
    int rc;
    if (nparticles > 0) {
      if ((rc = orc_set_new_particle(s, 0))) return rc;
      if ((rc = orc_calculate_trajectory(s))) return rc;
    } else if ((rc = ensure_trajectory(s))) return rc;
    double scale = fabs(s->p.q * s->p.current) / (16 * (K_PI * K_PI) * K_EPS0 * K_C);
    /* Result_Precision and Result_Level live outside the loop over facets (:3348-3349) */
    double result_precision = -1;
    int result_level = -1;
    for (long i = 0; i < n; ++i) {
      v3 obs = V(centers[3 * i], centers[3 * i + 1], centers[3 * i + 2]);
      v3 normal = V(tri[12 * i + 9], tri[12 * i + 10], tri[12 * i + 11]);
      double last_sum = -1, sum = 0;
      int last_level = 0;
      for (int L = 0; L <= lstop_ext; ++L) {
        last_level = L;
        v3 last_beta = V(0, 0, 0);
        double bdmax = -1;
        level_view lv;
        if (level_open(&s->tr, L, lstop_mem, &lv)) return fail(s, ORC_ERR_ALLOC, "alloc");
        for (long it = 0; it != lv.np; ++it) {
          double T; v3 X, B, A;
          level_point(&s->tr, &lv, it, &T, &X, &B, &A);
          int blocked = 0;
          for (long j = 0; j != n; ++j) {
            if (j == i) continue;
            v3 to = vsub(obs, X);
            double d = ray_intersection_distance(tri + 12 * j, X, vunit(to));
            if (d > 0 && d < vmag(to)) { blocked = 1; break; }
          }
          if (blocked) continue;
          double bd = vmag(vsub(B, last_beta));
          if (it > 0 && bd > bdmax) bdmax = bd;
          last_beta = B;
          v3 N1 = vunit(vsub(obs, X));
          v3 N2 = vunit(vorthogonal(N1));
          v3 N3 = vunit(vcross(N1, N2));
          double n1dn = fabs(vdot(N1, normal));
          v3 num = vcross(N1, vcross(vsub(N1, B), A));
          double den = pow(1 - vdot(B, N1), 5);
          double m2 = vmag2(vsub(obs, X));
          double d2 = vdot(num, N2), d3 = vdot(num, N3);
          sum += pow(d2, 2) / den / m2 * n1dn;
          sum += pow(d3, 2) / den / m2 * n1dn;
        }
        double ts = sum * delta_t_inclusive(&s->tr, L);
        result_precision = fabs(ts - last_sum) / last_sum;
        if ((L > 8 && result_precision < precision && bdmax < 2. / s->p.gamma) ||
            (L > 8 && bdmax < 2. / s->p.gamma && ts == last_sum)) {
          result_level = L;
          break;
        } else if (L > 8 && ts == last_sum) {
          result_level = L;
          result_precision = 0;
          break;
        }
        last_sum = ts;
      }
      sum *= scale * delta_t_inclusive(&s->tr, last_level);
      sum /= 1e6;
      double v;
      switch (quantity) {
        case 1: v = result_precision * weight; break;
        case 2: v = ((double)result_level) * weight; break;
        default: v = sum * weight; break;
      }
      out[i] = v + out[i];  /* TTriangle3D::AddToValue */
      if (out_level) out_level[i] = result_level;
    }
  }
  return ORC_OK;
}
