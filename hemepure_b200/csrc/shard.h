// shard.h -- one slab of a lattice for the sharded form (one lattice over several GPUs).
//
// The reference partitions a lattice over MPI ranks
// (src/geometry/decomposition/BasicDecomposition.cc:42-64 and the ParMETIS
// refinement) and, every step, sends the post-collision values of the links
// that cross into another rank's sites and copies the received values into
// place (src/geometry/LatticeData.cc:665-689).  Here a lattice is cut into slabs
// across one axis.  A shard's tables hold its own sites, in the reference's
// contiguous order, followed by the halo sites: the fluid sites of the plane
// just below and just above the slab.  The layout (layout.cpp) stores the halo
// sites after the owned ones and turns every push from a halo site into an
// owned site into a pull from the halo site's storage; the halo lists below say
// which (site, direction) values cross each cut.
#pragma once

#include <cstdint>
#include <vector>

#include "config.h"
#include "layout.h"

namespace hb {

// Slab bounds with balanced site counts: shard k owns the sites whose
// coordinate along *axis lies in [bounds[k], bounds[k+1]).  *axis < 0 picks the
// axis with the largest extent of fluid sites.
std::vector<int64_t> plan_slabs(const LatticeTables& t, int n_shards, int* axis);

// The tables of the shard owning [lo, hi) along `axis`: owned sites, then halo
// sites, each in the reference's contiguous order, with `gid` holding every
// site's global contiguous index and a neighbour table local to the shard.
// Rejects (HB_ERR_UNSUPPORTED) a Windkessel iolet whose sites or centre site lie
// in more than one shard: its flow sum would need a reduction across shards.
LatticeTables cut_shard(const LatticeTables& full, const hb_params& p, int axis, int64_t lo, int64_t hi);

// The values crossing the two cuts of a shard each step, as element indices
// i * np + storage index into a distribution buffer, in exchange order: sorted
// by (global site index, direction).  send[0] / recv[0] face the lower
// neighbour (coordinates below lo), send[1] / recv[1] the upper one.  A value
// sent is the post-collision f*_i of an owned site next to the cut whose link i
// pushes into the neighbour's slab; a value received is the same for a halo
// site, read by the owned site it pushes into.  The pairs (global index,
// direction) of each list are returned beside the element indices.
struct HaloLists {
  std::vector<int64_t> send[2], recv[2];
  std::vector<int64_t> send_pairs[2], recv_pairs[2];  // [2 * count]: global index, direction
};
HaloLists halo_lists(const LatticeTables& t, const Layout& L, int axis, int64_t lo, int64_t hi);

}  // namespace hb
