// layout.h -- device layout of one lattice, built on the host from the
// reference-order tables.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/hemeb200.h"
#include "config.h"

namespace hb {

struct Layout {
  int n = 0;                      // sites updated here (a shard's own sites)
  int n_halo = 0;                 // halo sites of a shard, stored at [n, n + n_halo)
  int64_t np = 0;                 // padded stride of one direction plane (covers the halo sites)
  int axis = 2;                   // run axis
  std::vector<int> st2ref, ref2st;
  std::vector<int> meta;          // [n]
  std::vector<int> run_off;       // [runs*20]
  int runs = 0;
  int bulk_sites = 0;
  // general sites (structure of arrays)
  int G = 0;
  std::vector<int> g_site, g_run, g_src, g_io, g_cpl, g_xyz, g_kind;
  int regular_general = 0;        // general sites whose bulk slots follow their run
  std::vector<uint32_t> g_wall, g_iolet;
  std::vector<float> g_q, g_nrm;
  int kind_start[7] = {0, 0, 0, 0, 0, 0, 0};   // bins by collision type
  // Windkessel coupling slots (reference order within each iolet)
  struct Coupling {
    int iolet = -1;               // table index (inlets 0..15, outlets 16..31)
    int start = 0, count = 0;
    int centre_ref = -1;
    bool centre_couples = false;
  };
  std::vector<Coupling> couplings; // one per WK3 iolet
  int cpl_total = 0;
  int dir0[32];
};

// Builds the layout; throws hb::Error (HB_ERR_UNSUPPORTED / HB_ERR_BAD_INDEX) for
// lattices whose streaming pattern the pull form cannot reproduce exactly.
Layout build_layout(const LatticeTables& t, const hb_params& p, int wall);

// The part of the layout that follows the general records (shared by the host
// and the device builds): record bins, Windkessel couplings and centre sites,
// the directions closest to the iolet normals, the GZS neighbour check.
void finish_layout(Layout& L, const LatticeTables& t, const hb_params& p, int wall);

// Lattice tables resident on the device (LatticeTables' fields, device pointers;
// q and normal may be null).
struct DeviceTables {
  int64_t n = 0;
  int64_t n_owned = -1;
  int64_t dims[3] = {0, 0, 0};
  const int64_t* coords = nullptr;
  const uint32_t* wall = nullptr;
  const uint32_t* iolet = nullptr;
  const int32_t* stype = nullptr;
  const int32_t* iolet_id = nullptr;
  const float* q = nullptr;
  const float* normal = nullptr;
};

// build_layout's passes up to the general records run on the GPU
// (layout_device.cu) over tables already on the device, on `stream`; the
// result is downloaded and equals build_layout's bit for bit once
// finish_layout has run on it.  Neighbours come from the coordinates.
Layout layout_on_device(const DeviceTables& d, const hb_params& p, void* stream);
// The same from host tables (uploaded first).  Tables that carry their own
// neighbour table are laid out on the host.
Layout build_layout_on_device(const LatticeTables& t, const hb_params& p, int wall, int device);

// FNV-1a digests of the layout's scalars and arrays (hb_geometry_layout_digest).
void layout_digest(const Layout& L, uint64_t out[32]);

// Direction closest to an iolet normal (SortDirectionsCloseToIOletNormal,
// src/lb/streamers/NashZerothOrderPressureDelegate.h:95-116).
int closest_direction(const double n[3]);

}  // namespace hb
