/*
 * hb_oracle.h -- CPU oracle for the D3Q19 collide-and-stream step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * single-rank algorithm (push form, reference site order, reference
 * arithmetic order).  Only the tests, the smoke check and the CPU-baseline leg
 * of the benchmark may load it, and only as the checker or the timed CPU
 * baseline.  The product library never links or calls it.
 */
#ifndef HB_ORACLE_H
#define HB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_Q = 19 };

/* Collision kernels (src/lb/kernels/LBGK.h, TRT.h, LBGKLESSpongeLayer.h). */
enum { ORC_LBGK = 0, ORC_TRT = 1, ORC_LBGKLES = 2, ORC_LBGKSL = 3, ORC_TRTSL = 4 };
/* Wall streamers (SimpleBounceBackDelegate.h, BouzidiFirdaousLallemandDelegate.h, GuoZhengShiDelegate.h). */
enum { ORC_SBB = 0, ORC_BFL = 1, ORC_GZS = 2 };
/* Iolet streamers and iolet value sources. */
enum { ORC_IOLET_COSINE = 0, ORC_IOLET_WK3 = 1, ORC_IOLET_PARABOLIC = 2, ORC_IOLET_WK2 = 3, ORC_IOLET_FILE = 4,
       ORC_IOLET_FILE_VELOCITY = 5, ORC_IOLET_WOMERSLEY = 6 };

typedef struct orc_iolet {
  int kind;                 /* ORC_IOLET_* */
  double position[3];       /* lattice units */
  double normal[3];         /* normalised, double (InOutLet::SetNormal) */
  /* cosine */
  double density_mean, density_amp, phase, period;
  uint64_t warmup;
  /* parabolic */
  double radius, max_speed;
  /* WK3 (lattice units); WK2 uses rp as its R and cp as its C */
  double rc, rp, cp, area;
  /* file pressure: density per 0-indexed step (InOutLetFile densityTable) and its minimum;
   * file velocity: peak speed per 1-based step (InOutLetFileVelocity velocityTable) */
  const double* table;
  uint64_t table_len;
  double density_min;
  /* Womersley: pressure-gradient amplitude and Womersley number (period, radius above) */
  double pressure_gradient_amplitude, womersley_number;
} orc_iolet;

typedef struct orc_params {
  int kernel, wall;
  double tau;                       /* LbmParameters tau */
  double relaxation_parameter;      /* TRT magic Lambda */
  double viscosity_ratio, sponge_width;
  uint64_t sponge_lifetime;
  double initial_density;
  uint64_t initial_step;            /* 1-based SimulationState time step */
  int n_inlets, n_outlets;
  orc_iolet inlets[16];
  orc_iolet outlets[16];
} orc_params;

typedef struct orc_lattice orc_lattice;
typedef struct orc_sim orc_sim;

/* Geometry + lattice construction (GeometryReader / LatticeData restated).
 * Returns 0 on success, a negative code on a malformed file. */
int orc_lattice_load(const char* gmy_path, orc_lattice** out, char* err, int errlen);
void orc_lattice_free(orc_lattice* lat);

int64_t orc_site_count(const orc_lattice* lat);
void orc_type_counts(const orc_lattice* lat, int64_t counts[6]);
void orc_dims(const orc_lattice* lat, int64_t blocks[3], int64_t* block_size);
/* Per-site tables in reference contiguous order. */
void orc_get_coords(const orc_lattice* lat, int64_t* xyz);            /* [N*3] */
void orc_get_neighbours(const orc_lattice* lat, int64_t* nbr);        /* [N*19] */
void orc_get_sitedata(const orc_lattice* lat, uint32_t* wall, uint32_t* iolet,
                      int32_t* type, int32_t* iolet_id);              /* [N] each */
void orc_get_wall_distance(const orc_lattice* lat, double* q);        /* [N*18] */
void orc_get_wall_normal(const orc_lattice* lat, double* n);          /* [N*3] */

/* Simulation. */
int orc_sim_create(const orc_lattice* lat, const orc_params* p, orc_sim** out, char* err, int errlen);
void orc_sim_free(orc_sim* s);
void orc_sim_set_threads(orc_sim* s, int nthreads);
/* Advance `steps` time steps.  If want_macro, the last step fills the density,
 * velocity and wall-shear-stress caches.  Returns 0, or 1 if unstable, or
 * negative on error (parabolic site outside the iolet radius). */
int orc_sim_run(orc_sim* s, int64_t steps, int want_macro);
uint64_t orc_sim_time_step(const orc_sim* s);
/* f_old (the distributions entering the next step), reference order, AoS [N*19]. */
void orc_sim_get_f(const orc_sim* s, double* f);
void orc_sim_set_f(orc_sim* s, const double* f);
void orc_sim_get_macro(const orc_sim* s, double* rho, double* u, double* wss);
/* Stress cache `field` of the last macro step (0 von Mises [n], 1 shear rate [n],
 * 2 stress tensor [n*6], 3 traction, 4 tangential, 5 normal projection [n*3]);
 * -1 before any macro step or for an unknown field. */
int orc_sim_get_stress(const orc_sim* s, int field, double* out);
/* WK3 state of iolet `index` of `group` (0 inlets, 1 outlets):
 * density, densityNew, flowRate, flowRateOld. */
void orc_sim_get_wk3(const orc_sim* s, int group, int index, double st[4]);
/* InOutLetVelocity::GetVelocity of a velocity iolet (parabolic, file velocity,
 * Womersley) at lattice position x and 1-based step t.  Returns 0, or -1 for a
 * point outside a parabolic or file profile's radius, -2 for a pressure iolet. */
int orc_iolet_velocity(const orc_iolet* io, const double x[3], uint64_t t, double v[3]);
/* util::BesselJ0ComplexArgument with tolSq = 1e-12 (src/util/Bessel.cc:17-43). */
void orc_bessel_j0(double re, double im, double out[2]);
/* Per-site relaxation time of the LES kernel's sponge layer (vTau). */
void orc_sim_get_vtau(const orc_sim* s, double* vtau);

#ifdef __cplusplus
}
#endif
#endif
