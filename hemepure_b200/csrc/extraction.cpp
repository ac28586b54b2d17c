// extraction.cpp -- .xtr v4 output, .off v1 offsets and checkpoint restore.
//
// Format (src/extraction/LocalPropertyOutput.cc:100-180, 217-365,
// src/io/formats/extraction.h, src/io/formats/offset.h), all XDR big-endian:
//   main header (60 B): hlb magic, 0x78747204, version 4, f64 voxel size,
//     3 x f64 origin, u64 site count, u32 field count, u32 field-header length;
//   per field: XDR string name, u32 floats per site, f64 offset;
//   per record: u64 time step, then per site in contiguous order u32 x, y, z and
//     the fields as f32 (pressure in mmHg minus the reference pressure, velocity
//     in m/s, shear stress in Pa, distributions in lattice units).
// A record labelled t carries the density/velocity/stress computed in step t and
// the distributions that entered step t (GetFNew after the swap,
// src/extraction/LbDataSourceIterator.cc:90-93).  The .off file holds the start
// of the first record and its end.
// Restore: src/extraction/LocalDistributionInput.cc:48-170 (binary search on the
// record labels, float values plus the field offset into f_old and f_new).
#include "extraction.h"

#include <sys/stat.h>

#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <vector>

#include "../../include/hemeb200.h"
#include "hb_common.h"
#include "solver.h"

namespace hb {

namespace {

constexpr uint32_t kHlbMagic = 0x686c6221u;
constexpr uint32_t kXtrMagic = 0x78747204u;
constexpr uint32_t kOffMagic = 0x6f666604u;
constexpr double kMmHgToPascal = 133.3223874;

struct XdrOut {
  std::vector<unsigned char> b;
  void u32(uint32_t v) {
    for (int k = 3; k >= 0; k--) b.push_back((unsigned char)(v >> (8 * k)));
  }
  void u64(uint64_t v) {
    u32((uint32_t)(v >> 32));
    u32((uint32_t)v);
  }
  void f32(float f) {
    uint32_t v;
    std::memcpy(&v, &f, 4);
    u32(v);
  }
  void f64(double d) {
    uint64_t v;
    std::memcpy(&v, &d, 8);
    u64(v);
  }
  void str(const std::string& s) {
    u32((uint32_t)s.size());
    for (char c : s) b.push_back((unsigned char)c);
    while (b.size() % 4) b.push_back(0);
  }
};

struct XdrIn {
  const unsigned char* p;
  size_t n, pos = 0;
  uint32_t u32() {
    if (pos + 4 > n) throw Error{HB_ERR_FORMAT, "truncated XDR data"};
    uint32_t v = (uint32_t(p[pos]) << 24) | (uint32_t(p[pos + 1]) << 16) | (uint32_t(p[pos + 2]) << 8) | uint32_t(p[pos + 3]);
    pos += 4;
    return v;
  }
  uint64_t u64() {
    uint64_t hi = u32();
    return (hi << 32) | u32();
  }
  float f32() {
    uint32_t v = u32();
    float f;
    std::memcpy(&f, &v, 4);
    return f;
  }
  double f64() {
    uint64_t v = u64();
    double d;
    std::memcpy(&d, &v, 8);
    return d;
  }
  std::string str() {
    uint32_t len = u32();
    if (pos + len > n) throw Error{HB_ERR_FORMAT, "truncated XDR string"};
    std::string s((const char*)p + pos, len);
    pos += len;
    while (pos % 4) pos++;
    return s;
  }
};

// Floats per site of each OutputField type (LocalPropertyOutput::GetFieldLength,
// src/extraction/LocalPropertyOutput.cc:367-391); 0 for an unknown type.
uint32_t field_len(const std::string& f) {
  if (f == "pressure" || f == "vonmisesstress" || f == "shearstress" || f == "shearrate" || f == "wallextension" ||
      f == "mpirank")
    return 1;
  if (f == "velocity" || f == "traction" || f == "tangentialprojectiontraction" || f == "normalprojectiontraction")
    return 3;
  if (f == "stresstensor") return 6;
  if (f == "distributions") return (uint32_t)Q;
  return 0;
}

// The stress cache an OutputField type reads, or -1.
int stress_field(const std::string& f) {
  if (f == "vonmisesstress") return HB_STRESS_VON_MISES;
  if (f == "shearrate") return HB_STRESS_SHEAR_RATE;
  if (f == "stresstensor") return HB_STRESS_TENSOR;
  if (f == "traction") return HB_STRESS_TRACTION;
  if (f == "tangentialprojectiontraction") return HB_STRESS_TANGENTIAL_TRACTION;
  if (f == "normalprojectiontraction") return HB_STRESS_NORMAL_TRACTION;
  return -1;
}

// Comma-separated entries "type" or "type:name" (the <field type= name=> of a
// <propertyoutput>; the name written in the header defaults to the type,
// SimConfig::DoIOForPropertyField, src/configuration/SimConfig.cc:566-580).
std::vector<std::string> split_fields(const std::string& s, std::vector<std::string>* names = nullptr) {
  std::vector<std::string> out;
  std::stringstream ss(s);
  std::string item;
  while (std::getline(ss, item, ',')) {
    size_t a = item.find_first_not_of(" \t"), b = item.find_last_not_of(" \t");
    if (a == std::string::npos) continue;
    item = item.substr(a, b - a + 1);
    std::string name = item;
    const size_t colon = item.find(':');
    if (colon != std::string::npos) {
      name = item.substr(colon + 1);
      item = item.substr(0, colon);
      if (name.empty()) throw Error{HB_ERR_ARG, "empty field name for type '" + item + "'"};
    }
    if (field_len(item) == 0) throw Error{HB_ERR_ARG, "Unrecognised field type '" + item + "'"};
    out.push_back(item);
    if (names) names->push_back(name);
  }
  if (out.empty()) throw Error{HB_ERR_ARG, "no output fields"};
  return out;
}


std::vector<unsigned char> read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error{HB_ERR_IO, "cannot open " + path};
  return std::vector<unsigned char>((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
}

// util::Vector3D<float> arithmetic of the reference's selectors: every operation
// rounds to float (the host build does not contract products into FMAs).
struct V3f {
  float x, y, z;
};
V3f sub(V3f a, V3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3f add(V3f a, V3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3f mul(V3f a, float k) { return {a.x * k, a.y * k, a.z * k}; }
V3f div(V3f a, float k) { return {a.x / k, a.y / k, a.z / k}; }
float dot(V3f a, V3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
float mag(V3f a) { return std::sqrt(dot(a, a)); }
V3f to_f(const double v[3]) { return {(float)v[0], (float)v[1], (float)v[2]}; }
V3f normalised(V3f v) {  // Vector3D::GetNormalised (util/Vector3D.h:270-292)
  if (v.x == 0.0f && v.y == 0.0f && v.z == 0.0f) return v;
  return div(v, mag(v));
}

}  // namespace

void selector_state(const hb_selector& sel, SelectArgs* a) {
  if (sel.type < HB_SELECT_WHOLE || sel.type > HB_SELECT_SURFACE_POINT) throw Error{HB_ERR_ARG, "unknown geometry selector"};
  const V3f point = to_f(sel.point), point2 = to_f(sel.point2);
  const V3f normal = normalised(to_f(sel.normal));
  const V3f line = sub(point2, point);
  a->type = sel.type;
  a->point[0] = point.x, a->point[1] = point.y, a->point[2] = point.z;
  a->normal[0] = normal.x, a->normal[1] = normal.y, a->normal[2] = normal.z;
  a->line[0] = line.x, a->line[1] = line.y, a->line[2] = line.z;
  a->radius = (float)sel.radius;
  a->line_len = mag(line);
  a->max_surface_dist = (float)std::sqrt(3.0);
}

std::vector<uint8_t> select_sites(const LatticeTables& t, const hb_selector& sel, double voxel, const double origin[3]) {
  const int64_t n = t.owned();  // a shard selects among its own sites
  std::vector<uint8_t> mask((size_t)n, 0);
  if (sel.type < HB_SELECT_WHOLE || sel.type > HB_SELECT_SURFACE_POINT) throw Error{HB_ERR_ARG, "unknown geometry selector"};
  // Selector state as the reference's constructors hold it: float vectors and radii.
  const V3f point = to_f(sel.point), point2 = to_f(sel.point2);
  const V3f normal = normalised(to_f(sel.normal));
  const float radius = (float)sel.radius;
  const V3f line = sub(point2, point);
  const float line_len = mag(line);
  const float max_surface_dist = (float)std::sqrt(3.0);
  for (int64_t i = 0; i < n; i++) {
    const bool wall = t.wall[i] != 0;
    // Vector3D<float>(location) * voxel + origin, in double, stored as float.
    const V3f c = {(float)((double)(float)t.coords[3 * i] * voxel + origin[0]),
                   (float)((double)(float)t.coords[3 * i + 1] * voxel + origin[1]),
                   (float)((double)(float)t.coords[3 * i + 2] * voxel + origin[2])};
    bool take = false;
    switch (sel.type) {
      case HB_SELECT_WHOLE:
        take = true;
        break;
      case HB_SELECT_PLANE: {
        const float perp = dot(sub(c, point), normal);
        if (std::abs(perp) > 0.5 * voxel) break;
        if (radius <= 0.) {
          take = true;
          break;
        }
        const float r2 = dot(sub(sub(c, mul(normal, perp)), point), sub(sub(c, mul(normal, perp)), point));
        take = r2 <= radius * radius;
        break;
      }
      case HB_SELECT_LINE: {
        const float along = dot(line, sub(c, point)) / line_len;
        if (along < 0. || along > line_len) break;
        const V3f d = sub(add(point, div(mul(line, along), line_len)), c);
        take = dot(d, d) <= 2.0 * 0.5 * 0.5 * voxel * voxel;
        break;
      }
      case HB_SELECT_SPHERE:
        take = mag(sub(c, point)) <= radius;
        break;
      case HB_SELECT_INLET:
        take = t.stype[i] == 1;
        break;
      case HB_SELECT_OUTLET:
        take = t.stype[i] == 2;
        break;
      case HB_SELECT_SURFACE:
        take = wall;
        break;
      case HB_SELECT_SURFACE_WITHIN_SPHERE:
        take = wall && mag(sub(c, point)) <= radius;
        break;
      case HB_SELECT_SURFACE_POINT: {
        if (!wall) break;
        const float d = (float)(mag(sub(c, point)) / voxel);
        take = d <= max_surface_dist;
        break;
      }
    }
    mask[(size_t)i] = take ? 1 : 0;
  }
  return mask;
}

void write_xtr(Solver& s, const std::string& path, const std::string& fields_csv, const std::string& offset_path,
               const hb_selector* sel) {
  std::vector<std::string> names;
  const std::vector<std::string> fields = split_fields(fields_csv, &names);
  const LatticeTables& t = s.tables();
  const int64_t n = t.owned();
  if (s.time_step() <= 1) throw Error{HB_ERR_ARG, "no completed time step to write"};
  const uint64_t label = s.time_step() - 1;
  bool need_macro = false, need_f = false, need_stress[6] = {false, false, false, false, false, false};
  for (auto& f : fields) {
    if (f == "distributions") need_f = true;
    else if (f == "pressure" || f == "velocity" || f == "shearstress") need_macro = true;
    const int sf = stress_field(f);
    if (sf >= 0) need_stress[sf] = true;
  }
  // Data per written site k (row k of each array), and the written sites'
  // indices in reference order.  With a selector, the sites are selected and
  // their data gathered on the device, and only they are downloaded.
  std::vector<int> idx;
  std::vector<double> rho, u, wss, fd;
  std::vector<double> stress[6];
  if (sel) {
    Solver::Selection got = s.select(*sel, need_macro, need_stress, need_f);
    idx = std::move(got.idx);
    rho = std::move(got.rho);
    u = std::move(got.u);
    wss = std::move(got.wss);
    fd = std::move(got.fd);
    for (int k = 0; k < 6; k++) stress[k] = std::move(got.stress[k]);
  } else {
    idx.resize(n);
    for (int64_t i = 0; i < n; i++) idx[i] = (int)i;
    for (int k = 0; k < 6; k++) {
      if (!need_stress[k]) continue;
      if (!s.stress_valid())
        throw Error{HB_ERR_ARG, "the last step did not fill the stress caches (pass HB_STEP_MACRO | HB_STEP_STRESS)"};
      stress[k].resize((size_t)n * Solver::stress_len(k));
      s.get_stress(k, stress[k].data());
    }
    if (need_macro) {
      if (!s.macro_valid()) throw Error{HB_ERR_ARG, "the last step did not fill the macroscopic caches (pass HB_STEP_MACRO)"};
      rho.resize(n);
      u.resize(3 * n);
      wss.resize(n);
      s.get_macro(rho.data(), u.data(), wss.data());
    }
    if (need_f) {
      fd.resize((size_t)n * Q);
      if (!s.get_previous_fs(fd.data())) throw Error{HB_ERR_ARG, "the distributions of the last step are no longer held"};
    }
  }
  const int64_t n_out = (int64_t)idx.size();

  // Unit conversion (src/util/UnitConverter.cc, UnitConverter.h:61-119).
  const double dx = s.dx(), dt = s.dt();
  const double mass = 1000.0 * dx * dx * dx;
  const double lattice_pressure = mass / (dx * dt * dt);
  const double lattice_speed = dx / dt;
  const double lattice_time = dt;
  // REFERENCE_PRESSURE_mmHg (src/constants.h:23), kept in the expressions so that
  // signed zeros and the non-finite normals of sites off the wall come out as the
  // reference's conversions give them.
  constexpr double kRefPressureMmHg = 0.0;
  const HostArray<float>& normal = t.normal;

  XdrOut hdr;
  {
    XdrOut fh;
    for (size_t k = 0; k < fields.size(); k++) {
      const std::string& f = fields[k];
      fh.str(names[k]);
      fh.u32(field_len(f));
      fh.f64(0.0);  // REFERENCE_PRESSURE_mmHg for pressure, 0 otherwise
    }
    hdr.u32(kHlbMagic);
    hdr.u32(kXtrMagic);
    hdr.u32(4);
    hdr.f64(dx);
    hdr.f64(s.origin()[0]);
    hdr.f64(s.origin()[1]);
    hdr.f64(s.origin()[2]);
    hdr.u64((uint64_t)n_out);
    hdr.u32((uint32_t)fields.size());
    hdr.u32((uint32_t)fh.b.size());
    hdr.b.insert(hdr.b.end(), fh.b.begin(), fh.b.end());
  }
  XdrOut rec;
  rec.u64(label);
  for (int64_t i = 0; i < n_out; i++) {
    const int64_t x = idx[i];  // the site's index in reference order; i is its row in the data arrays
    rec.u32((uint32_t)t.coords[3 * x]);
    rec.u32((uint32_t)t.coords[3 * x + 1]);
    rec.u32((uint32_t)t.coords[3 * x + 2]);
    for (auto& f : fields) {
      if (f == "pressure") {
        const double p = rho[i] * kCs2;
        rec.f32((float)(0.0 + (p - kCs2) * lattice_pressure / kMmHgToPascal - 0.0));
      } else if (f == "velocity") {
        rec.f32((float)(u[3 * i] * lattice_speed));
        rec.f32((float)(u[3 * i + 1] * lattice_speed));
        rec.f32((float)(u[3 * i + 2] * lattice_speed));
      } else if (f == "shearstress") {
        rec.f32((float)(wss[i] * lattice_pressure));
      } else if (f == "vonmisesstress") {
        // ConvertStressToPhysicalUnits (src/util/UnitConverter.h:61-64).
        rec.f32((float)(stress[HB_STRESS_VON_MISES][i] * lattice_pressure));
      } else if (f == "shearrate") {
        // ConvertShearRateToPhysicalUnits (src/util/UnitConverter.cc:48-52).
        rec.f32((float)(stress[HB_STRESS_SHEAR_RATE][i] / lattice_time));
      } else if (f == "stresstensor") {
        // ConvertFullStressTensorToPhysicalUnits (UnitConverter.h:73-78): the
        // upper triangle row by row, the reference pressure off the diagonal.
        const double* st = &stress[HB_STRESS_TENSOR][(size_t)i * 6];
        for (int k = 0; k < 6; k++) {
          double v = st[k] * lattice_pressure;
          if (k == 0 || k == 3 || k == 5) v += -kRefPressureMmHg * kMmHgToPascal;
          rec.f32((float)v);
        }
      } else if (f == "traction") {
        // ConvertTractionToPhysicalUnits (UnitConverter.h:90-96) with the site's
        // wall normal (non-finite off the wall, LatticeData.cc:242-244).
        const double* tr = &stress[HB_STRESS_TRACTION][(size_t)i * 3];
        const double scale = lattice_speed * lattice_speed * 1000.0;
        for (int k = 0; k < 3; k++) {
          const double nk = (double)normal[(size_t)3 * x + k];
          rec.f32((float)(tr[k] * scale - nk * kRefPressureMmHg * kMmHgToPascal));
        }
      } else if (f == "tangentialprojectiontraction" || f == "normalprojectiontraction") {
        const int sf = stress_field(f);
        for (int k = 0; k < 3; k++) rec.f32((float)(stress[sf][(size_t)i * 3 + k] * lattice_pressure));
      } else if (f == "wallextension") {
        // Rigid walls: no delegate here sets a wall extension (only the elastic
        // GZS delegate does, GuoZhengShiElasticWallDelegate.h:70), so it is 0.
        rec.f32((float)(0.0 * dx));
      } else if (f == "mpirank") {
        rec.f32((float)0);  // one rank
      } else {
        for (int k = 0; k < Q; k++) rec.f32((float)fd[(size_t)i * Q + k]);
      }
    }
  }

  struct stat sb;
  const bool exists = stat(path.c_str(), &sb) == 0 && sb.st_size > 0;
  if (exists) {
    std::vector<unsigned char> old = read_file(path);
    if (old.size() < hdr.b.size() || std::memcmp(old.data(), hdr.b.data(), hdr.b.size()) != 0)
      throw Error{HB_ERR_FORMAT, "existing .xtr file has a different header"};
    if ((old.size() - hdr.b.size()) % rec.b.size() != 0) throw Error{HB_ERR_FORMAT, "existing .xtr file has a partial record"};
    std::ofstream out(path, std::ios::binary | std::ios::app);
    out.write((const char*)rec.b.data(), (std::streamsize)rec.b.size());
    if (!out) throw Error{HB_ERR_IO, "cannot append to " + path};
  } else {
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    out.write((const char*)hdr.b.data(), (std::streamsize)hdr.b.size());
    out.write((const char*)rec.b.data(), (std::streamsize)rec.b.size());
    if (!out) throw Error{HB_ERR_IO, "cannot write " + path};
  }
  if (!offset_path.empty()) {
    XdrOut off;
    off.u32(kHlbMagic);
    off.u32(kOffMagic);
    off.u32(1);
    off.u32(1);
    off.u64((uint64_t)hdr.b.size());
    off.u64((uint64_t)(hdr.b.size() + rec.b.size()));
    std::ofstream out(offset_path, std::ios::binary | std::ios::trunc);
    out.write((const char*)off.b.data(), (std::streamsize)off.b.size());
    if (!out) throw Error{HB_ERR_IO, "cannot write " + offset_path};
  }
}

void read_checkpoint(Solver& s, const std::string& path, uint64_t step) {
  std::vector<unsigned char> buf = read_file(path);
  XdrIn x{buf.data(), buf.size()};
  if (x.u32() != kHlbMagic) throw Error{HB_ERR_FORMAT, "This file does not start with the HemeLB magic number."};
  if (x.u32() != kXtrMagic) throw Error{HB_ERR_FORMAT, "This file is not an extraction file."};
  if (x.u32() != 4) throw Error{HB_ERR_FORMAT, "Unsupported extraction version."};
  x.f64();
  x.f64();
  x.f64();
  x.f64();
  const uint64_t nsites = x.u64();
  const uint32_t nfields = x.u32();
  const uint32_t fhl = x.u32();
  (void)fhl;
  if (nfields != 1) throw Error{HB_ERR_FORMAT, "a checkpoint holds exactly one field"};
  const std::string name = x.str();
  const uint32_t nf = x.u32();
  const double offset = x.f64();
  if (name != "distributions" || nf != (uint32_t)Q) throw Error{HB_ERR_FORMAT, "checkpoint field is not 'distributions' of 19 values"};
  const LatticeTables& t = s.tables();
  if ((int64_t)nsites != t.owned()) throw Error{HB_ERR_FORMAT, "checkpoint site count differs from the lattice"};
  const size_t hdr = x.pos;
  const size_t reclen = 8 + (size_t)nsites * (12 + 4 * Q);
  if ((buf.size() - hdr) % reclen != 0) throw Error{HB_ERR_FORMAT, "Checkpoint file length not consistent with integer number of checkpoints"};
  const size_t ntimes = (buf.size() - hdr) / reclen;
  if (ntimes == 0) throw Error{HB_ERR_FORMAT, "checkpoint file holds no record"};
  auto label_of = [&](size_t k) {
    XdrIn r{buf.data() + hdr + k * reclen, 8};
    return r.u64();
  };
  size_t idx = ntimes - 1;
  if (step) {
    size_t lo = 0, len = ntimes;
    while (len) {
      size_t half = len / 2, m = lo + half;
      if (label_of(m) < step) {
        lo = m + 1;
        len -= half + 1;
      } else {
        len = half;
      }
    }
    if (lo >= ntimes || label_of(lo) != step) throw Error{HB_ERR_ARG, "Target timestep not found in checkpoint file."};
    idx = lo;
  }
  XdrIn r{buf.data() + hdr + idx * reclen, reclen};
  const uint64_t label = r.u64();
  std::vector<double> f((size_t)t.owned() * Q);
  for (int64_t i = 0; i < t.owned(); i++) {
    const uint32_t px = r.u32(), py = r.u32(), pz = r.u32();
    if ((int64_t)px != t.coords[3 * i] || (int64_t)py != t.coords[3 * i + 1] || (int64_t)pz != t.coords[3 * i + 2])
      throw Error{HB_ERR_FORMAT, "Site read at index " + std::to_string(i) + " does not match the lattice's site order"};
    for (int k = 0; k < Q; k++) {
      float v = r.f32();
      v = (float)((double)v + offset);
      f[(size_t)i * Q + k] = (double)v;
    }
  }
  s.set_fs(f.data());
  s.set_time_step(label);
}

}  // namespace hb
