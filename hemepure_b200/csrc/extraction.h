// extraction.h -- .xtr property output and checkpoint restore
// (src/extraction/LocalPropertyOutput.cc, src/extraction/LocalDistributionInput.cc).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/hemeb200.h"

namespace hb {

class Solver;
struct LatticeTables;

struct SelectArgs;

// Sites an extraction geometry selector takes (src/extraction/*Selector.cc), as
// a mask over the lattice in contiguous order; voxel size and origin in metres.
std::vector<uint8_t> select_sites(const LatticeTables& t, const hb_selector& sel, double voxel, const double origin[3]);
// The selector's state as the reference's constructors hold it (float vectors
// and radii, the normal normalised in float), for the device selector kernel.
void selector_state(const hb_selector& sel, SelectArgs* out);

// Append one output record for the sites `sel` takes (the whole lattice when null).
void write_xtr(Solver& s, const std::string& path, const std::string& fields, const std::string& offset_path,
               const hb_selector* sel = nullptr);
// Restore f_old = f_new from the "distributions" record with time `step`
// (0 = the last record), then set the time step to that record's label.
void read_checkpoint(Solver& s, const std::string& path, uint64_t step);

}  // namespace hb
