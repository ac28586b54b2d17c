// device.h -- device-side data layout shared by the host driver and the kernels.
//
// Layout in HBM (one lattice):
//   f_a, f_b   [19][np] distributions, structure of arrays, ping-pong.  After a
//              step the output buffer holds POST-collision values f*(x) (pull
//              form); before the first step it holds PRE-collision f (direct form).
//   meta       [n]  run id of a plain bulk site, or -(g+1) for general site g.
//   run_off    [runs][20] per-direction source offset of a plain bulk site:
//              slot i of site s is pulled from f*[i][s + run_off[run][i]].
//   general    per general site (wall, iolet, or bulk sites whose neighbours do
//              not follow the run pattern), structure of arrays, binned by
//              collision type so a warp runs one streamer.
//   ghost_a/b  [18][G] iolet ghost values (Nash / Ladd) of general site g for
//              link d, ping-pong with f: slot inv(d) of the next step reads them.
#pragma once

#include <cstdint>

namespace hb {

struct IoletDev {
  int kind;               // IoletKind
  int dir0;               // direction closest to the iolet normal
  int wk3;                // index into the Windkessel state, or -1
  int pad;
  double pos[3];
  double nrm[3];          // normalised normal (double)
  double nrm_f[3];        // the normal narrowed to float and widened back (Nash ghost)
  double radius, max_speed;
  uint64_t warmup;
};

struct WK3Dev {           // InOutLetWK3 / InOutLetWK2 state
  double density, density_new, flow, flow_old;
  double rc, rp, cp, area;    // WK2: rp is R, cp is C
  int cpl_start, cpl_count;   // coupling slots of this iolet
  int count_prev;             // coupling sites summed at the previous step (0 before the first)
  int centre_couples;         // the centre site takes part in the coupling
  int iolet;                  // index into the iolet table
  int kind;                   // kWK3 or kWK2
  int pad[2];
};

// What a step launcher launches (`which`): the plain bulk sites, all boundary
// records, or the boundary records without iolet links or those with them, for
// launching the two on separate streams.
constexpr int kLaunchBulk = 1, kLaunchBoundary = 2, kLaunchWallRecords = 4, kLaunchIoletRecords = 8;

struct GeneralDev {
  int G;
  int G_noiolet;          // records [0, G_noiolet) have no iolet links (the first two collision-type bins)
  const int* site;        // [G] storage index
  const int* run;         // [G] run whose offsets the bulk slots follow, or -1
  const uint32_t* wall;   // [G] wall-link mask (bit d-1 for direction d)
  const uint32_t* iolet;  // [G] iolet-link mask
  const int* src;         // [18][G] pull source of slots 1..18 when run < 0
  const float* q;         // [18][G] wall distances (BFL, GZS)
  const float* nrm;       // [3][G] wall normal (float, normalised in float)
  const int* io;          // [G] iolet table index or -1
  const int* cpl;         // [G] Windkessel coupling slot or -1
  const int* xyz;         // [3][G] global coordinates
  const int* wom;         // [G] row of a Womersley iolet site in StepArgs::wom_amp, or -1 (null without one)
};

struct StepArgs {
  const double* fin;
  double* fout;
  const double* gin;      // iolet ghost values produced with fin [18][G]
  double* gout;           // iolet ghost values of this step [18][G]
  int64_t np;
  int n;
  const int* meta;
  const int* run_off;
  const int* run_po;      // [runs][20] plane offsets i * np + run_off[run][i] (shifted forms' bulk kernel), or null
  GeneralDev gen;
  // kernel parameters
  double tau, omega, omega_minus;
  double lambda;          // TRT magic parameter (TRTSL: per-site omega_minus)
  const double* vtau;     // LES sponge tau per site (storage order) or null
  uint64_t t;             // 1-based time step of this step
  uint64_t lifetime;      // LES sponge lifetime
  const IoletDev* iolets;
  const double* dens_row; // this step's iolet row [kRowStride]: densities, then velocity-iolet values
  const double* wom_amp;  // [K][18][4] Womersley factor A of link d of Womersley site k:
                          // (Re, Im) at the half-way point x + c_d / 2, then at x + c_d
  double* cpl_buf;        // Windkessel coupling contributions
  double* rho;            // macroscopic outputs in storage order (or null)
  double* u;              // [3][np]
  double* wss;
  int* status;            // bit 0 unstable, bit 1 iolet radius, bit 2 bad neighbour
  // Output steps that need the stress caches: the non-equilibrium momentum flux
  // tensor (xx, xy, xz, yy, yz, zz) and the relaxation time of each site, [7][np];
  // null otherwise.
  double* pi;
};

// One row of per-step iolet values: the density of iolet idx (inlets 0-15,
// outlets 16-31) at [idx]; for a file-velocity iolet its peak speed at
// [kRowA + idx]; for a Womersley iolet Re and Im of exp(i omega t) at
// [kRowA + idx] and [kRowB + idx].
constexpr int kRowA = 32, kRowB = 64, kRowStride = 96;

enum StatusBits { kStatusUnstable = 1, kStatusIoletRadius = 2, kStatusBadNeighbour = 4 };

// Launchers (kernels_f64.cu).
// `which`: 1 = plain bulk sites, 2 = general sites, 3 = both.
void launch_step_f64(const StepArgs& a, int kernel, int wall, bool gather, bool macro, int which, int bulk_block,
                     int general_block, void* stream);
void launch_gather_f64(const StepArgs& a, int wall, void* stream);
// Gather the pre-collision f straight into AoS reference order.
void launch_gather_aos_f64(const StepArgs& a, int wall, const int* st2ref, double* aos, void* stream);
// Stress caches in lattice units from StepArgs::pi and rho of an output step
// (BaseStreamer::UpdateMinsAndMaxes, src/lb/streamers/BaseStreamer.h:123-217):
// field HB_STRESS_*, `out` [k][np] in storage order, k the field's length.
void launch_stress_field(const StepArgs& a, int field, double* out, void* stream);
void launch_wk3_begin(WK3Dev* wk3, int nwk3, const double* cpl_buf, double* dens_row, void* stream);
void launch_equilibrium_f64(double* f, int64_t np, int n, const double feq[19], void* stream);
void launch_equilibrium_aos_f64(double* f, int n, const double feq[19], void* stream);
// Shifted low-precision storage (kernels_mixed.cu): g = f - w stored as FP32, or
// as FP16 holding g * kHalfScale; ghosts in FP32.
void launch_step_mixed(const StepArgs& a, int precision, const void* fin, void* fout, const float* gin, float* gout,
                       int kernel, int wall, bool gather, bool macro, int which, void* stream);
void launch_to_aos_mixed(const StepArgs& a, int precision, const void* fin, const float* gin, int wall, bool gather,
                         const int* st2ref, double* aos, void* stream);
void launch_from_aos_mixed(const double* aos, const int* st2ref, int n, int64_t np, int precision, void* out, void* stream);
// Conserved sums (density, momentum x/y/z) over n sites in FP64, deterministic:
// one partial per block of kSumSitesPerBlock sites in `scratch` (4 doubles per
// block), then the partials in block order into `out` (4 doubles, device).
constexpr int kSumThreads = 256;
constexpr int kSumSitesPerBlock = 2048;
int moment_sum_blocks(int64_t n);
void launch_moment_sums(const double* f, int64_t dir_stride, int64_t site_stride, int64_t n, double* scratch,
                        double* out, void* stream);
// Extraction on the device (extract.cu): a geometry selector evaluated per site
// in the reference's order, in the reference selectors' float arithmetic.
struct SelectArgs {
  int64_t n;
  const int32_t* coords;   // [n*3] lattice coordinates, reference order
  const uint8_t* wall;     // [n] 1 for a site with a wall link
  const uint8_t* stype;    // [n] 0 fluid, 1 inlet, 2 outlet
  double voxel, origin[3];
  int type;                // HB_SELECT_*
  float point[3], normal[3], line[3];
  float radius, line_len, max_surface_dist;
};
int select_blocks(int64_t n);
// mask[n] and the selected indices in reference order into idx (*total of them);
// counts needs select_blocks(n) ints.
void launch_select(const SelectArgs& s, uint8_t* mask, int* counts, int* total, int* idx, void* stream);
// out[k*width + j] = src[j*stride + ref2st[idx[k]]] for k < m (a field in storage order).
void launch_gather_selected(const double* src, int64_t stride, int width, const int* idx, const int* ref2st, int m,
                            double* out, void* stream);
// out[k*width + j] = aos[idx[k]*width + j] (rows of an array in reference order).
void launch_gather_rows(const double* aos, int width, const int* idx, int m, double* out, void* stream);
// Sharded form (shard.cu): out[k] = f[idx[k]] and f[idx[k]] = in[k] over m
// stored elements of `elem_bytes` bytes (8 FP64, 4 FP32, 2 FP16 storage).
void launch_halo_pack(const void* f, const int64_t* idx, int64_t m, void* out, int elem_bytes, void* stream);
void launch_halo_unpack(const void* in, const int64_t* idx, int64_t m, void* f, int elem_bytes, void* stream);
// AoS reference order <-> SoA storage order.
void launch_soa_to_aos_f64(const double* soa, int64_t np, const int* st2ref, int n, double* aos, void* stream);
void launch_aos_to_soa_f64(const double* aos, const int* st2ref, int n, double* soa, int64_t np, void* stream);

}  // namespace hb
