// extraction.h -- .xtr property output and checkpoint restore
// (src/extraction/LocalPropertyOutput.cc, src/extraction/LocalDistributionInput.cc).
#pragma once

#include <cstdint>
#include <string>

namespace hb {

class Solver;

// Append one output record for the whole lattice.
void write_xtr(Solver& s, const std::string& path, const std::string& fields, const std::string& offset_path);
// Restore f_old = f_new from the "distributions" record with time `step`
// (0 = the last record), then set the time step to that record's label.
void read_checkpoint(Solver& s, const std::string& path, uint64_t step);

}  // namespace hb
