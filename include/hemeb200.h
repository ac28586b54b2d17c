/*
 * hemeb200.h -- C ABI of the B200 D3Q19 collide-and-stream library (libhemeb200.so).
 *
 * The library replaces the per-time-step work of the reference's lb::LBM
 * (src/lb/lb.h:32-148, src/lb/lb.hpp:119-346): the six streamers run over the
 * type-contiguous site ranges in PreSend/PreReceive, the post-step fix-ups in
 * PostReceive and the swap in EndIteration.  Everything the reference keeps in
 * geometry::LatticeData for that path (distributions, neighbour indices, site
 * data, wall distances and normals; src/geometry/LatticeData.h:624-653) lives in
 * device memory behind an opaque handle.
 *
 * All functions return an int status: HB_OK (0) on success, a positive value for
 * a numerical condition (HB_UNSTABLE), a negative value for an error.  Nothing
 * throws across the ABI.  Site-indexed host arrays are in the reference's
 * contiguous site order (collision types 0..5, each in block-traversal order),
 * and distributions are AoS [site*19 + direction] doubles, exactly as the
 * reference stores f_old/f_new.  One host thread per handle.
 */
#ifndef HEMEB200_H
#define HEMEB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (reference: hemelb::Exception / SimulationState::SetStability) */
#define HB_OK 0
#define HB_UNSTABLE 1            /* some f <= 0 or NaN (src/lb/StabilityTester.h:100-111) */
#define HB_ERR_ARG (-1)          /* bad argument or handle */
#define HB_ERR_IO (-2)           /* file cannot be read or written */
#define HB_ERR_FORMAT (-3)       /* malformed XML / .gmy / .xtr */
#define HB_ERR_CUDA (-4)         /* a CUDA call failed */
#define HB_ERR_OOM (-5)          /* device memory exhausted */
#define HB_ERR_BAD_INDEX (-6)    /* a site or neighbour table failed validation */
#define HB_ERR_UNSUPPORTED (-7)  /* configuration outside the supported set */
#define HB_ERR_IOLET_RADIUS (-8) /* parabolic or file-velocity iolet point outside its radius (reference exit(16)) */
#define HB_ERR_TIMEOUT (-9)      /* a bounded device wait gave up */

/* ---- run-time selectable types (reference: compile-time CMake strings,
 *      src/CMakeLists.txt:43-65, src/lb/BuildSystemInterface.h:24-369) */
#define HB_KERNEL_LBGK 0         /* src/lb/kernels/LBGK.h */
#define HB_KERNEL_TRT 1          /* src/lb/kernels/TRT.h */
#define HB_KERNEL_LBGKLESSL 2    /* src/lb/kernels/LBGKLESSpongeLayer.h */
#define HB_KERNEL_LBGKSL 3       /* src/lb/kernels/LBGKSpongeLayer.h (FP64 storage) */
#define HB_KERNEL_TRTSL 4        /* src/lb/kernels/TRTSpongeLayer.h (FP64 storage) */

#define HB_WALL_SBB 0            /* src/lb/streamers/SimpleBounceBackDelegate.h */
#define HB_WALL_BFL 1            /* src/lb/streamers/BouzidiFirdaousLallemandDelegate.h */
#define HB_WALL_GZS 2            /* src/lb/streamers/GuoZhengShiDelegate.h */

#define HB_IOLET_COSINE 0        /* Nash pressure, src/lb/iolets/InOutLetCosine.cc */
#define HB_IOLET_WK3 1           /* Nash pressure, src/lb/iolets/InOutLetWK3.cc */
#define HB_IOLET_PARABOLIC 2     /* Ladd velocity, src/lb/iolets/InOutLetParabolicVelocity.cc */
#define HB_IOLET_WK2 3           /* Nash pressure, src/lb/iolets/InOutLetWK2.cc (R in rp, C in cp) */
#define HB_IOLET_FILE 4          /* Nash pressure from a time-pressure file, src/lb/iolets/InOutLetFile.cc */
#define HB_IOLET_FILE_VELOCITY 5 /* Ladd velocity, parabolic profile whose peak follows a time-speed file,
                                    src/lb/iolets/InOutLetFileVelocity.cc */
#define HB_IOLET_WOMERSLEY 6     /* Ladd velocity, Womersley profile, src/lb/iolets/InOutLetWomersleyVelocity.cc */

/* ---- where the .gmy site records are decoded (same tables either way) */
#define HB_GEOMETRY_HOST 0       /* one host thread (GeometryReader's steps) */
#define HB_GEOMETRY_DEVICE 1     /* inflate on host threads, decode, order and link on the GPU */

/* ---- storage precision of the distributions */
#define HB_STORE_FP64 0          /* plain form: FP64 storage and arithmetic */
#define HB_STORE_FP32 1          /* f - w_i rho0 stored in FP32, FP32 collision */
#define HB_STORE_FP16 2          /* f - w_i rho0 stored in FP16, FP32 collision */

/* ---- hb_step flags */
#define HB_STEP_MACRO 1u         /* fill density, velocity and wall-shear-stress on the last step */
#define HB_STEP_STRESS 2u        /* with HB_STEP_MACRO: also fill the stress caches (hb_get_stress) */

/* ---- stress caches (MacroscopicPropertyCache, src/lb/MacroscopicPropertyCache.h) */
#define HB_STRESS_VON_MISES 0            /* [n]   vonMisesStressCache */
#define HB_STRESS_SHEAR_RATE 1           /* [n]   shearRateCache */
#define HB_STRESS_TENSOR 2               /* [n*6] stressTensorCache: xx, xy, xz, yy, yz, zz */
#define HB_STRESS_TRACTION 3             /* [n*3] tractionCache (zero off the wall) */
#define HB_STRESS_TANGENTIAL_TRACTION 4  /* [n*3] tangentialProjectionTractionCache */
#define HB_STRESS_NORMAL_TRACTION 5      /* [n*3] normalProjectionTractionCache */

typedef struct hb_handle hb_handle;

typedef struct hb_options {
  int kernel;     /* HB_KERNEL_* (the reference's HEMELB_KERNEL) */
  int wall;       /* HB_WALL_* (the reference's HEMELB_WALL_BOUNDARY) */
  int precision;  /* HB_STORE_* */
  int device;     /* CUDA device ordinal */
  int geometry_reader; /* HB_GEOMETRY_*: where hb_create_from_xml decodes the .gmy */
} hb_options;

/* One inlet or outlet in lattice units (reference: iolets::InOutLet and subclasses). */
typedef struct hb_iolet {
  int kind;                 /* HB_IOLET_* */
  double position[3];       /* InOutLet::GetPosition */
  double normal[3];         /* normalised; points into the fluid (InOutLet::SetNormal) */
  double density_mean, density_amp, phase, period; /* cosine (InOutLetCosine); period also Womersley */
  uint64_t warmup;          /* extra_warmup_steps */
  double radius, max_speed; /* parabolic (InOutLetParabolicVelocity); radius also file velocity, Womersley */
  double rc, rp, cp, area;  /* WK3 (InOutLetWK3); WK2 and fileWK (InOutLetWK2, InOutLetFileWK) use rp as R, cp as C */
  /* file iolets: one value per step, indexed as the reference indexes its table (steps
   * beyond it take its last entry).  File pressure (InOutLetFile): the lattice density
   * per 0-indexed step (its densityTable), with the table's minimum density.  File
   * velocity (InOutLetFileVelocity): the lattice peak speed per 1-based step (its
   * velocityTable).  The library copies the table when a handle is created;
   * hb_read_case leaves it NULL (hb_read_case_iolet_table fills a caller buffer). */
  const double* table;
  uint64_t table_steps;
  double density_min;
  /* Womersley (InOutLetWomersleyVelocity): pressure-gradient amplitude (lattice units),
   * Womersley number; the period is `period`, the radius `radius`. */
  double pressure_gradient_amplitude, womersley_number;
} hb_iolet;

/* LbmParameters + iolet set + initial condition, all in lattice units. */
typedef struct hb_params {
  double tau;                   /* LbmParameters::GetTau (src/lb/LbmParameters.h:29-37) */
  double relaxation_parameter;  /* TRT magic number (SimConfig relaxation_parameter) */
  double viscosity_ratio;       /* LES sponge layer */
  double sponge_width;          /* lattice units */
  uint64_t sponge_lifetime;
  double initial_density;       /* equilibrium initial condition (InitialCondition.cc:71-73) */
  uint64_t initial_step;        /* 1-based SimulationState time step */
  int n_inlets, n_outlets;
  hb_iolet inlets[16];
  hb_iolet outlets[16];
} hb_params;

/* The lattice as the reference's LatticeData holds it after
 * LatticeData::ProcessReadSites / InitialiseNeighbourLookup on one rank. */
typedef struct hb_lattice_desc {
  int64_t n_sites;
  int64_t dims[3];              /* global lattice extent in sites */
  const int64_t* coords;        /* [n*3] GetGlobalSiteCoords */
  const uint32_t* wall_mask;    /* [n] SiteData::GetWallIntersectionData */
  const uint32_t* iolet_mask;   /* [n] SiteData::GetIoletIntersectionData */
  const int32_t* site_type;     /* [n] 0 fluid, 1 inlet, 2 outlet (geometry::SiteType) */
  const int32_t* iolet_id;      /* [n] SiteData::GetIoletId */
  const double* wall_distance;  /* [n*18] GetCutDistance(site, 1..18); may be NULL for SBB */
  const double* wall_normal;    /* [n*3] GetNormalToWall; may be NULL */
  const int64_t* neighbours;    /* [n*19] neighbourIndices, or NULL to derive from coords */
} hb_lattice_desc;

/* ---- construction / teardown ------------------------------------------- */

/* Default options: LBGK, SBB, FP64, device 0. */
void hb_default_options(hb_options* opt);

/* Build from a case file: SimConfig::New (src/configuration/SimConfig.cc:41-121),
 * GeometryReader::LoadAndDecompose (src/geometry/GeometryReader.cc:63-365),
 * new LatticeData, LBM ctor + Initialise + SetInitialConditions. */
int hb_create_from_xml(const char* xml_path, const hb_options* opt, hb_handle** out);

/* Build from lattice tables the caller already holds (the drop-in path: the
 * reference keeps its GeometryReader/LatticeData and hands the tables over). */
int hb_create(const hb_lattice_desc* lat, const hb_params* params, const hb_options* opt, hb_handle** out);

int hb_destroy(hb_handle* h);

/* Last error message of this handle (or of the last failed create when h is NULL). */
int hb_last_error(const hb_handle* h, char* msg, size_t len);

/* ---- lb::LBM per-step phases (src/lb/lb.hpp:191-346) ------------------------ */

/* BeginPhase: LBM::RequestComms + BoundaryValues::RequestComms (no halo on one GPU;
 * Windkessel state advances on the device). */
int hb_request_comms(hb_handle* h);
/* LBM::PreSend: domain-edge sites; none on one GPU, kept for the call sequence. */
int hb_pre_send(hb_handle* h);
/* LBM::PreReceive: collide and stream every site (all six collision types). */
int hb_pre_receive(hb_handle* h, uint32_t flags);
/* LBM::PostReceive: the post-step fix-ups are folded into the next gather. */
int hb_post_receive(hb_handle* h);
/* LBM::EndIteration + SimulationState::Increment. */
int hb_end_iteration(hb_handle* h);

/* All phases of `n_steps` time steps; HB_STEP_MACRO fills the caches on the last.
 * A shard (below) advances one step per call. */
int hb_step(hb_handle* h, int64_t n_steps, uint32_t flags);

/* ---- exact restart in FP64 ------------------------------------------------------
 * No counterpart in the reference, whose checkpoint is the float32
 * "distributions" field of an .xtr file (LocalDistributionInput,
 * src/extraction/LocalDistributionInput.cc:48-298; hb_read_checkpoint reads it),
 * so a restart from it is not the run that would have continued.  This state
 * file holds the distributions entering the next step in FP64, the time step,
 * and each Windkessel iolet's state with the coupling contributions its next
 * flow sum reads: a run restored from it continues bit for bit.  FP64 storage
 * only (HB_ERR_UNSUPPORTED otherwise); the restore checks that the file's sites
 * are the handle's, in the same order (HB_ERR_FORMAT otherwise). */
int hb_write_state(hb_handle* h, const char* path);
int hb_read_state(hb_handle* h, const char* path);

/* ---- one lattice over several GPUs: slabs with a halo exchange --------------
 * The reference decomposes a lattice over MPI ranks
 * (src/geometry/decomposition/BasicDecomposition.cc:42-64, refined by
 * OptimisedDecomposition) and every step sends the post-collision values of
 * the links crossing into another rank and copies the received ones into place
 * (LatticeData::SendAndReceive / CopyReceived, src/geometry/LatticeData.cc:665-689).
 * Here the lattice is cut into slabs across one axis, one per GPU.  A shard
 * handle owns its slab's sites and keeps the fluid sites of the plane beyond
 * each cut as halo sites.  After each hb_step(h, 1, ...) the caller packs the
 * values its two neighbours pull (hb_shard_pack), exchanges the buffers with
 * them (for example NCCL send/recv), and unpacks what it received
 * (hb_shard_unpack) before the next step.  Each list is ordered by (global
 * site index, direction), so neighbouring shards agree on it without talking.
 * The arithmetic of every site is the single-lattice arithmetic: the shards
 * together give the single-lattice results bit for bit.  Rejected with
 * HB_ERR_UNSUPPORTED: a GZS wall link whose extrapolation neighbour is a halo
 * site, and a Windkessel iolet whose sites or centre site span two slabs. */
typedef struct hb_shard {
  int axis;       /* 0, 1 or 2: the axis the cuts cross */
  int64_t lo, hi; /* this shard owns the sites with lo <= coordinate < hi */
} hb_shard;

/* Slab bounds with balanced site counts for n_shards shards: shard k owns
 * [bounds[k], bounds[k+1]); *axis < 0 on entry picks the axis with the largest
 * extent of fluid sites (the axis is returned).  bounds has n_shards + 1 entries.
 * Plays the role of BasicDecomposition::Decompose for slabs. */
int hb_shard_plan(const char* xml_path, int kernel, int n_shards, int* axis, int64_t* bounds);
/* hb_create_from_xml for one shard. */
int hb_create_shard_from_xml(const char* xml_path, const hb_options* opt, const hb_shard* shard, hb_handle** out);
/* Stored elements sent to the lower / upper neighbour and received from them
 * per step: counts[0] send lower, [1] send upper, [2] receive lower, [3]
 * receive upper; *elem_bytes: 8 (FP64), 4 (FP32) or 2 (FP16 storage). */
int hb_shard_halo_sizes(const hb_handle* h, int64_t counts[4], int* elem_bytes);
/* After a step: the values the neighbours pull, into device buffers of
 * counts[0] and counts[1] elements (NULL where the count is 0).  Ordered after
 * the step on the handle's stream; `stream` (a cudaStream_t, or NULL) is made to
 * wait for the pack, so work queued on it afterwards sees the buffers filled. */
int hb_shard_pack(hb_handle* h, void* to_lower, void* to_upper, void* stream);
/* Before the next step: the neighbours' values into the halo sites.  The unpack
 * waits for the work queued so far on `stream` (where the receives completed). */
int hb_shard_unpack(hb_handle* h, const void* from_lower, const void* from_upper, void* stream);
/* Global contiguous index of each owned site, in the handle's reference order
 * (the order of hb_get_fs and hb_get_macro), [n]. */
int hb_shard_site_ids(const hb_handle* h, int64_t* ids);
/* The same shard described on the host, with no GPU: counts[0] owned sites,
 * [1] halo sites, [2..5] entries of the send-lower, send-upper, receive-lower and
 * receive-upper lists; owned / halo: global indices; each list: (global site
 * index, direction) pairs in exchange order.  Any output pointer may be NULL. */
int hb_shard_describe(const char* xml_path, int kernel, int wall, const hb_shard* shard, int64_t counts[6],
                      int64_t* owned, int64_t* halo, int64_t* send_lower, int64_t* send_upper, int64_t* recv_lower,
                      int64_t* recv_upper);

/* ---- state access ---------------------------------------------------------- */

int hb_site_count(const hb_handle* h, int64_t* n);
int hb_time_step(const hb_handle* h, uint64_t* t);          /* 1-based, as SimulationState */
/* Set the time step of the next step (InitialCondition::SetTime, src/lb/InitialCondition.cc:18-21). */
int hb_set_time_step(hb_handle* h, uint64_t t);
int hb_get_params(const hb_handle* h, hb_params* p);         /* LBM::GetLbmParams + iolets */
/* f_old in reference order, AoS [n*19] (LatticeData::GetFOld after EndIteration). */
int hb_get_fs(hb_handle* h, double* f);
/* Replace f_old and f_new (InitialCondition / checkpoint restore). */
int hb_set_fs(hb_handle* h, const double* f);
/* MacroscopicPropertyCache of the last HB_STEP_MACRO step: density [n], velocity
 * [n*3], wall-shear-stress magnitude [n] (NO_VALUE = DBL_MAX off the wall).
 * Any pointer may be NULL. */
int hb_get_macro(hb_handle* h, double* density, double* velocity, double* wss);
/* Stress cache `field` (HB_STRESS_*) of the last HB_STEP_MACRO | HB_STEP_STRESS step,
 * in lattice units and reference order, as BaseStreamer::UpdateMinsAndMaxes fills
 * it (src/lb/streamers/BaseStreamer.h:123-217; Lattice.h:983-1180): the von Mises
 * stress and shear rate of the non-equilibrium momentum flux tensor, the full stress
 * tensor -Pi - (rho - 1) cs^2 I, and at wall sites the traction sigma.n with its
 * tangential and normal projections. */
int hb_get_stress(hb_handle* h, int field, double* out);
/* BoundaryValues::GetBoundaryDensity supplied by the caller (the per-step iolet
 * values of src/lb/iolets/BoundaryValues.cc:211-214, for a HemePure host that keeps
 * its own iolet objects or couples them to another model): lattice densities of
 * every inlet and outlet, in the case's order, used by the cosine and file pressure
 * iolets from the next step on in place of their own GetDensity (no warm-up blend);
 * Windkessel densities stay on the device and velocity iolets ignore theirs.  The
 * counts must be the case's; both pointers NULL returns to the case's values. */
int hb_set_iolet_densities(hb_handle* h, const double* inlet_density, int n_inlets, const double* outlet_density,
                           int n_outlets);
/* Total density and momentum (x, y, z) of the distributions entering the next
 * step, summed in FP64 in a fixed order: the per-step mass and flux balance
 * the reference's monitoring computes on the host (src/lb/IncompressibilityChecker.hpp). */
int hb_moment_sums(hb_handle* h, double sums[4]);
/* Windkessel state of iolet `index` of `group` (0 inlets, 1 outlets):
 * density, densityNew, flowRate, flowRateOld (InOutLetWK3 members). */
int hb_get_wk3(hb_handle* h, int group, int index, double state[4]);

/* Integer tables in reference order, for bit-exact comparison with the reference:
 * neighbourIndices [n*19], wall and iolet masks [n], site type [n], iolet id [n],
 * coords [n*3], per-type site counts [6] (any pointer may be NULL). */
int hb_get_tables(const hb_handle* h, int64_t* neighbours, uint32_t* wall_mask, uint32_t* iolet_mask,
                  int32_t* site_type, int32_t* iolet_id, int64_t* coords, int64_t* type_counts);

/* ---- extraction and checkpoint (src/extraction/) ---------------------------- */

/* Write one .xtr output step (LocalPropertyOutput::Write, float32 XDR) for the
 * whole lattice with the listed fields (comma-separated OutputField types:
 * "pressure", "velocity", "shearstress", "vonmisesstress", "shearrate",
 * "stresstensor", "traction", "tangentialprojectiontraction",
 * "normalprojectiontraction", "wallextension", "distributions", "mpirank", each
 * optionally "type:name" to write the field under a name of its own;
 * the stress types need the step run with HB_STEP_STRESS).  Appends a record if the file exists with
 * a matching header; `offset_path` (may be NULL) receives the .off file. */
int hb_write_xtr(hb_handle* h, const char* path, const char* fields, const char* offset_path);
/* Extraction geometry selectors (the <geometry type=...> of a <propertyoutput>,
 * SimConfig::DoIOForPropertyOutputFile, src/configuration/SimConfig.cc:421-484):
 * whole lattice; plane through `point` with `normal` (within half a voxel of it,
 * and within `radius` of `point` when radius > 0); straight line from `point` to
 * `point2`; sphere of `radius` about `point`; inlet or outlet sites; wall sites;
 * wall sites in the sphere; wall sites within sqrt(3) voxels of `point`.  Points
 * and radii in metres; the tests are made in the reference's float arithmetic
 * (src/extraction/PlaneGeometrySelector.cc:54-81, StraightLineGeometrySelector.cc:30-49,
 * SphereGeometrySelector.cc, SurfacePointSelector.cc:22-40). */
enum {
  HB_SELECT_WHOLE = 0,
  HB_SELECT_PLANE = 1,
  HB_SELECT_LINE = 2,
  HB_SELECT_SPHERE = 3,
  HB_SELECT_INLET = 4,
  HB_SELECT_OUTLET = 5,
  HB_SELECT_SURFACE = 6,
  HB_SELECT_SURFACE_WITHIN_SPHERE = 7,
  HB_SELECT_SURFACE_POINT = 8
};
typedef struct hb_selector {
  int type;
  double point[3];
  double point2[3];
  double normal[3];
  double radius;
} hb_selector;
/* hb_write_xtr restricted to the sites `sel` takes (header site count included). */
int hb_write_xtr_selected(hb_handle* h, const char* path, const char* fields, const char* offset_path,
                          const hb_selector* sel);
/* Restore f from the "distributions" field of an .xtr at time step `step`
 * (LocalDistributionInput::LoadDistribution). */
int hb_read_checkpoint(hb_handle* h, const char* path, uint64_t step);

/* ---- batched form: many lattices of uneven size on one GPU ------------------------ */

/* The batched form keeps many independent lattices resident in one device arena
 * (shifted FP32 or FP16 storage) and steps them together: per step one
 * persistent kernel over every member's plain bulk sites and one over every
 * member's boundary sites, with per-lattice relaxation times, iolets and time
 * counters in device memory, the steps of a block captured once in a CUDA graph.
 * Members are admitted and retired between blocks without moving the others.
 * Supported per member: LBGK or TRT, bounce-back or BFL walls, cosine pressure
 * and parabolic velocity iolets.  Capacities: sites (rounded to 64 per member),
 * boundary records, member slots. */
typedef struct hb_batch hb_batch;
int hb_batch_bytes(int64_t site_capacity, int64_t general_capacity, int max_lattices, int precision, int64_t* bytes);
int hb_batch_create(int64_t site_capacity, int64_t general_capacity, int max_lattices, int precision, int device,
                    hb_batch** out);
int hb_batch_destroy(hb_batch* b);
/* Admit a lattice for `steps` time steps; returns its slot.  HB_ERR_OOM when it does not fit. */
int hb_batch_add_xml(hb_batch* b, const char* xml_path, int kernel, int wall, uint64_t steps, int* slot);
int hb_batch_add(hb_batch* b, const hb_lattice_desc* lat, const hb_params* params, int kernel, int wall, uint64_t steps,
                 int* slot);
int hb_batch_remove(hb_batch* b, int slot);
/* The host half of hb_batch_add_xml, for overlapping admission with running
 * blocks: parse the case, read the geometry, check the physics is supported and
 * build the storage layout.  Needs no device, touches no batch, and may run on
 * any number of threads at once.  hb_batch_add_prepared then only uploads; on
 * HB_OK the batch has taken the prepared lattice's contents, on any error (e.g.
 * HB_ERR_OOM, no room yet) they stay for a later attempt.  The caller frees the
 * object with hb_batch_prep_free either way. */
typedef struct hb_batch_prep hb_batch_prep;
int hb_batch_prepare_xml(const char* xml_path, int kernel, int wall, uint64_t steps, hb_batch_prep** out);
/* The same with the site records decoded and the storage layout built on
 * `device` (the result is identical).  Its device allocations and frees
 * synchronise that device, so a server preparing while a batch steps on the
 * same device keeps to hb_batch_prepare_xml. */
int hb_batch_prepare_xml_device(const char* xml_path, int kernel, int wall, uint64_t steps, int device,
                                hb_batch_prep** out);
int hb_batch_prep_sites(const hb_batch_prep* prep, int64_t* sites);
int hb_batch_add_prepared(hb_batch* b, hb_batch_prep* prep, int* slot);
int hb_batch_prep_free(hb_batch_prep* prep);
/* Run a block of k steps; the slots that reached their step count, or went
 * unstable during the block (status bits set; such a member stops stepping and
 * its macroscopic fields are not filled), are written to
 * finished[0 .. *n_finished) (at most max_finished). */
int hb_batch_run(hb_batch* b, int k, int* finished, int max_finished, int* n_finished);
/* Density [n], velocity [n*3], wall shear stress [n] of a finished member's last step, reference order. */
int hb_batch_get_macro(hb_batch* b, int slot, double* density, double* velocity, double* wss);
/* Member sites, time step reached, status bits (1 unstable, 2 iolet radius). */
int hb_batch_member_info(hb_batch* b, int slot, int64_t* sites, uint64_t* time_step, int* status);
/* Sites per thread (1, 2) and threads per block (128, 256) of the bulk kernel. */
int hb_batch_set_tuning(hb_batch* b, int sites_per_thread, int block);
/* Form of the step kernel: one persistent kernel interleaving bulk and boundary
 * tiles (HB_BATCH_STEP_PERSISTENT, the default), or the same tiles as two ordinary
 * kernels run side by side (HB_BATCH_STEP_SPLIT).  A tuning choice; results are
 * identical. */
#define HB_BATCH_STEP_PERSISTENT 0
#define HB_BATCH_STEP_SPLIT 1
int hb_batch_set_step_form(hb_batch* b, int form);
/* Device time of the last block in ms, active sites, device bytes held. */
int hb_batch_stats(const hb_batch* b, double* last_block_ms, int64_t* active_sites, int64_t* device_bytes);

/* ---- host-only readers (no GPU needed) ------------------------------------------ */

/* SimConfig::DoIO for the collide-and-stream path: lattice-unit parameters and
 * the geometry path (resolved against the case file's directory). */
int hb_read_case(const char* xml_path, int kernel, hb_params* params, char* gmy_path, size_t gmy_path_len);
/* The table of a file iolet of a case (`outlet` 0 for inlets, 1 for outlets; `index`
 * within the group): densities of a file-pressure iolet, peak speeds of a
 * file-velocity iolet; its first `count` entries. */
int hb_read_case_iolet_table(const char* xml_path, int kernel, int outlet, int index, double* out, uint64_t count);

/* InOutLetVelocity::GetVelocity of a velocity iolet (parabolic, file velocity or
 * Womersley) at lattice position x and 1-based time step t, evaluated on the host in
 * the reference's FP64 arithmetic; the kernels impose exactly these values on the
 * Ladd links.  A parabolic or file-velocity iolet returns HB_ERR_IOLET_RADIUS for a
 * point outside its radius (the reference exits there); a pressure iolet returns
 * HB_ERR_UNSUPPORTED.  Replaces the iolet's own GetVelocity (for example
 * src/lb/iolets/InOutLetWomersleyVelocity.cc:25-41). */
int hb_iolet_velocity(const hb_iolet* iolet, const double x[3], uint64_t t, double v[3]);

typedef struct hb_geometry hb_geometry;
/* GeometryReader + LatticeData on one rank: the reference-order tables. */
int hb_geometry_open(const char* gmy_path, hb_geometry** out);
/* The same tables (bit for bit) with the site records decoded, binned into the
 * contiguous order and linked into the neighbour table on GPU `device`; the
 * blocks are inflated on a pool of host threads. */
int hb_geometry_open_device(const char* gmy_path, int device, hb_geometry** out);
/* Wall-clock milliseconds of the last open's phases: file read and header,
 * inflate, host-to-device copy, device decode/order/link, device-to-host copy
 * (host reader: all of it in ms[0]). */
int hb_geometry_read_timing(const hb_geometry* g, double ms[5]);
int hb_geometry_site_count(const hb_geometry* g, int64_t* n, int64_t dims[3]);
/* Same arrays as hb_get_tables plus wall distances [n*18] and normals [n*3]. */
int hb_geometry_tables(const hb_geometry* g, int64_t* neighbours, uint32_t* wall_mask, uint32_t* iolet_mask,
                       int32_t* site_type, int32_t* iolet_id, int64_t* coords, int64_t* type_counts,
                       double* wall_distance, double* wall_normal);
/* Device layout summary without allocating: run axis, runs, plain bulk sites,
 * general sites (or an error if the lattice cannot be streamed exactly). */
int hb_geometry_layout(const hb_geometry* g, const hb_params* params, int wall, int64_t stats[4]);
/* FNV-1a digests of every array and scalar of the storage layout, built on the
 * host (device < 0) or on that device: [0] scalars (n, halo, stride, axis, runs,
 * bulk and general counts, bins, coupling total, closest directions), [1..16]
 * st2ref, ref2st, meta, run offsets, and the general records' site, run,
 * sources, iolet, coupling slot, coordinates, kind, wall and iolet masks,
 * cut distances, normals, couplings; the rest 0.  Both builds give the same
 * digests for every lattice (a check of the device passes). */
int hb_geometry_layout_digest(const hb_geometry* g, const hb_params* params, int wall, int device, uint64_t digest[32]);
/* The selector's site mask over the geometry (contiguous order; 1 = taken), for a
 * voxel size and origin in metres.  Host-only. */
int hb_geometry_select(const hb_geometry* g, const hb_selector* sel, double voxel_size, const double origin[3],
                       uint8_t* mask);
int hb_geometry_close(hb_geometry* g);

/* ---- without device allocation --------------------------------------------------- */

/* Total density and momentum (x, y, z) of n_sites sites, like hb_moment_sums but
 * on device buffers the caller owns, for callers whose device memory is all
 * committed elsewhere (their own pool or a fixed HBM budget) and who must not
 * have the library allocate.  No reference counterpart: the reference sums on
 * the host.  Distribution i of site s is f[i*dir_stride + s*site_stride] (FP64,
 * device); the four sums go to `sums` (device) on `stream` (a cudaStream_t, or
 * NULL).  Nothing is allocated: the scratch is a fixed 256 KiB array in the
 * library, so one call takes at most 16,777,216 sites (more returns HB_ERR_ARG).
 * The first call on a device looks up that array's device address (once per
 * device, again after a device reset replaced the device's context); make it
 * before any stream capture.  Under CUDA's lazy module loading (the default)
 * the array is created on a device when the library's module loads there, at
 * the latest by that first call: a caller that commits all its device memory
 * makes one warm-up call before.  Calls share the array, so two calls whose
 * kernels overlap on one GPU race; the result is ready when `stream` is
 * synchronised.  Errors: hb_last_error(NULL, ...). */
int hb_moment_sums_noalloc(const double* f, int64_t dir_stride, int64_t site_stride, int64_t n_sites, double* sums,
                           void* stream);

/* ---- measurement helpers ----------------------------------------------------- */

/* Device-time of the last hb_step call's kernels in milliseconds (CUDA events),
 * and the number of kernel launches it made. */
int hb_last_step_timing(const hb_handle* h, double* ms, int64_t* launches);
/* Replaces the set-up timers of reporting::Timers (fileRead, unzip,
 * latDatInitialise; src/reporting/Timers.h:82-100).
 * Wall-clock milliseconds of hb_create_from_xml's phases: ms[0] the case file,
 * ms[1] the geometry (with the device reader: decode, layout and the tables'
 * copy back), ms[2] the solver (uploads, initial state), ms[3] the total;
 * zeros for a handle made another way. */
int hb_setup_timing(const hb_handle* h, double ms[4]);
/* Advance 2 x `n_steps` steps with CUDA events around the launches (for
 * measurement only).  The first n_steps run as hb_step runs them and ms[0]
 * sums their collide-and-stream launch (one fused kernel, or the bulk and
 * boundary kernels side by side); the next n_steps run the plain-bulk kernel
 * and then the boundary kernel, and ms[1] and ms[2] sum those. */
int hb_profile_steps(hb_handle* h, int64_t n_steps, double ms[3]);
/* Bytes of device memory held by the handle. */
int hb_device_bytes(const hb_handle* h, int64_t* bytes);

#ifdef __cplusplus
}
#endif
#endif /* HEMEB200_H */
