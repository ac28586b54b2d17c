// config.cpp -- XML v3 case reader and .gmy v4 geometry reader for one rank.
//
// Case file: src/configuration/SimConfig.cc:84-198 (simulation), 262-408 (iolets),
// 640-655 (iolet position/normal), 668-723 (initial conditions, sponge),
// 725-754 (cosine), 756-794 (file, WK2), 796-824 (WK3), 826-854 (fileWK),
// 856-876 (parabolic), 878-901 (Womersley), 937-954 (file velocity); the file
// iolets' tables src/lb/iolets/InOutLetFile.cc:48-127 and
// InOutLetFileVelocity.cc:34-101; velocity profiles InOutLetParabolicVelocity.cc,
// InOutLetFileVelocity.cc:104-128, InOutLetWomersleyVelocity.cc:25-41 with
// src/util/Bessel.cc:17-43; unit conversion
// src/util/UnitConverter.cc:15-118 and UnitConverter.h:153-203; tau from
// src/lb/LbmParameters.h:29-37.
//
// Geometry: src/geometry/GeometryReader.cc:382-444 (preamble), 515-607 (header),
// 800-946 (inflate, site records); classification src/geometry/SiteDataBare.cc:24-172;
// site order src/geometry/LatticeData.cc:69-285 and LatticeData.h:375-436;
// neighbour table src/geometry/LatticeData.cc:366-443.
#include <sys/mman.h>

#include <cstdlib>
#include "config.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>

#include "xml.h"

namespace hb {

namespace {

constexpr double kMmHgToPascal = 133.3223874;
constexpr double kBloodDensity = 1000.0;
constexpr double kBloodViscosity = 0.004;

double parse_double(const std::string& s, const std::string& what) {
  char* end = nullptr;
  double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str()) throw Error{HB_ERR_FORMAT, "cannot parse number '" + s + "' for " + what};
  return v;
}

uint64_t parse_u64(const std::string& s, const std::string& what) {
  char* end = nullptr;
  unsigned long long v = std::strtoull(s.c_str(), &end, 10);
  if (end == s.c_str()) throw Error{HB_ERR_FORMAT, "cannot parse integer '" + s + "' for " + what};
  return (uint64_t)v;
}

void parse_vec(const std::string& s, double out[3], const std::string& what) {
  // "(x,y,z)"
  size_t a = s.find('('), b = s.rfind(')');
  if (a == std::string::npos || b == std::string::npos || b <= a) throw Error{HB_ERR_FORMAT, "bad vector '" + s + "' for " + what};
  std::string body = s.substr(a + 1, b - a - 1);
  size_t c1 = body.find(','), c2 = body.find(',', c1 == std::string::npos ? 0 : c1 + 1);
  if (c1 == std::string::npos || c2 == std::string::npos) throw Error{HB_ERR_FORMAT, "bad vector '" + s + "' for " + what};
  out[0] = parse_double(body.substr(0, c1), what);
  out[1] = parse_double(body.substr(c1 + 1, c2 - c1 - 1), what);
  out[2] = parse_double(body.substr(c2 + 1), what);
}

// GetDimensionalValue: checks the units attribute, then reads "value".
const std::string& dim_value(const XmlElement& el, const std::string& units) {
  const std::string& got = el.attr("units");
  if (got != units)
    throw Error{HB_ERR_FORMAT, "Invalid units for element " + el.name + ". Expected '" + units + "', got '" + got + "'"};
  return el.attr("value");
}

struct Units {
  double dx, dt, mass, speed, pressure;
  Units(double dt_, double dx_) : dx(dx_), dt(dt_) {
    mass = kBloodDensity * dx * dx * dx;
    speed = dx / dt;
    pressure = mass / (dx * dt * dt);
  }
  double pressure_diff(double dp) const { return dp * kMmHgToPascal / pressure; }
  double pressure_abs(double p) const { return kCs2 + pressure_diff(p - 0.0); }
  double to_lattice(const std::string& u, double v) const {
    double sf;
    if (u == "m") sf = dx;
    else if (u == "s") sf = dt;
    else if (u == "rad" || u == "dimensionless") sf = 1.;
    else if (u == "m/s") sf = dx / dt;
    else if (u == "mmHg") sf = mass / (dx * dt * dt) / kMmHgToPascal;
    else if (u == "mmHg/m") sf = mass / (dx * dx * dt * dt) / kMmHgToPascal;
    else throw Error{HB_ERR_FORMAT, "Unknown units '" + u + "'"};
    return v / sf;
  }
};

// util::NumericalFunctions::LinearInterpolate (src/util/utilityFunctions.h:96-134).
double linear_interpolate(const std::vector<double>& xs, const std::vector<double>& ys, double x) {
  size_t i = 0;
  while (!(x >= xs[i] && x <= xs[i + 1])) {
    i++;
    if (i + 1 >= xs.size()) throw Error{HB_ERR_FORMAT, "file iolet: interpolation beyond the file's time range"};
  }
  return ys[i] + (x - xs[i]) / (xs[i + 1] - xs[i]) * (ys[i + 1] - ys[i]);
}

// The read loop and end-of-run clipping shared by InOutLetFile::CalculateTable
// (src/lb/iolets/InOutLetFile.cc:48-98) and InOutLetFileVelocity::CalculateTable
// (src/lb/iolets/InOutLetFileVelocity.cc:34-76): (time in s, value) pairs in
// time order, cut at total_steps * dt with an interpolated last pair.
void read_profile(const std::string& path, uint64_t total_steps, double dt, std::vector<double>& times,
                  std::vector<double>& values) {
  std::ifstream in(path);
  if (!in) throw Error{HB_ERR_IO, "cannot open iolet file " + path};
  std::map<double, double> pairs;
  double t = 0.0, v = 0.0;
  while (in.good()) {  // the reference's read loop, with its end-of-file behaviour
    in >> t >> v;
    pairs[t] = v;
  }
  const double end = (double)total_steps * dt;
  for (const auto& e : pairs) {
    if (e.first > end) {
      if (times.empty()) throw Error{HB_ERR_FORMAT, "file iolet: the file starts after the simulation ends"};
      const double ratio = (end - times.back()) / (e.first - times.back());
      const double final_v = values.back() + ratio * (e.second - values.back());
      times.push_back(end);
      values.push_back(final_v);
      break;
    }
    times.push_back(e.first);
    values.push_back(e.second);
  }
}

// Both tables loop the file's profile with the same (odd) point formula:
// point = t_first + ((ts mod steps in the profile) / total_steps) * (t_last - t_first).
template <class F>
void profile_table(const std::vector<double>& times, const std::vector<double>& values, uint64_t total_steps,
                   double dt, std::vector<double>& table, F to_lattice) {
  const int period = (int)(times.back() / dt);
  if (period <= 0 || total_steps == 0) throw Error{HB_ERR_FORMAT, "file iolet: the file spans less than one step"};
  table.resize(total_steps + 1);
  for (uint64_t ts = 0; ts <= total_steps; ts++) {
    const double point =
        times.front() + ((double)(ts % (uint64_t)period) / (double)total_steps) * (times.back() - times.front());
    table[ts] = to_lattice(linear_interpolate(times, values, point));
  }
}

// InOutLetFile::CalculateTable: the lattice density at every step 0..total_steps
// from a file of (time in s, pressure in mmHg) pairs, and the minimum density.
void file_density_table(const std::string& path, uint64_t total_steps, double dt, const Units& u,
                        std::vector<double>& table, double& density_min) {
  std::vector<double> times, values;
  read_profile(path, total_steps, dt, times, values);
  density_min = u.pressure_abs(*std::min_element(values.begin(), values.end())) / kCs2;
  profile_table(times, values, total_steps, dt, table, [&](double p) { return u.pressure_abs(p) / kCs2; });
}

// InOutLetFileVelocity::CalculateTable: the lattice peak speed at every step
// 0..total_steps from a file of (time in s, speed in m/s) pairs
// (UnitConverter::ConvertVelocityToLatticeUnits divides by voxel / time step).
void file_velocity_table(const std::string& path, uint64_t total_steps, double dt, const Units& u,
                         std::vector<double>& table) {
  std::vector<double> times, values;
  read_profile(path, total_steps, dt, times, values);
  profile_table(times, values, total_steps, dt, table, [&](double v) { return v / u.speed; });
}

void normalise(double n[3]) {
  if (n[0] == 0.0 && n[1] == 0.0 && n[2] == 0.0) return;
  const double m = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] /= m;
  n[1] /= m;
  n[2] /= m;
}

}  // namespace

CaseConfig read_case(const std::string& xml_path, int kernel) {
  auto root = xml_parse_file(xml_path);
  CaseConfig c;
  if (root->name != "hemelbsettings") throw Error{HB_ERR_FORMAT, "Invalid root element: " + root->name};
  if (parse_u64(root->attr("version"), "version") != 3)
    throw Error{HB_ERR_FORMAT, "Unrecognised XML version. Expected 3, got " + root->attr("version")};
  const XmlElement& sim = root->require("simulation");
  c.total_steps = parse_u64(dim_value(sim.require("steps"), "lattice"), "steps");
  c.dt = parse_double(dim_value(sim.require("step_length"), "s"), "step_length");
  if (const XmlElement* wu = sim.child("extra_warmup_steps")) {
    c.warmup = parse_u64(dim_value(*wu, "lattice"), "extra_warmup_steps");
    c.total_steps += c.warmup;
  }
  hb_params& p = c.params;
  std::memset(&p, 0, sizeof(p));
  if (kernel == kTRT || kernel == kTRTSL)  // SimConfig.cc:165
    p.relaxation_parameter = parse_double(dim_value(sim.require("relaxation_parameter"), "lattice"), "relaxation_parameter");
  c.dx = parse_double(dim_value(sim.require("voxel_size"), "m"), "voxel_size");
  parse_vec(dim_value(sim.require("origin"), "m"), c.origin, "origin");
  Units u(c.dt, c.dx);
  p.tau = 0.5 + (c.dt * kBloodViscosity / kBloodDensity) / (kCs2 * c.dx * c.dx);

  std::string gmy = root->require("geometry").require("datafile").attr("path");
  if (!gmy.empty() && gmy[0] != '/') {
    size_t slash = xml_path.rfind('/');
    if (slash != std::string::npos) gmy = xml_path.substr(0, slash + 1) + gmy;
  }
  c.gmy_path = gmy;

  const XmlElement& ic = root->require("initialconditions");
  p.initial_step = 1;
  if (const XmlElement* te = ic.child("time")) {
    p.initial_step = parse_u64(dim_value(*te, "lattice"), "time");
    c.has_time = true;
  }
  const XmlElement* pe = ic.child("pressure");
  const XmlElement* ce = ic.child("checkpoint");
  if (pe && ce) throw Error{HB_ERR_FORMAT, "XML contains both <pressure> and <checkpoint> sub elements of <initialconditions>"};
  if (!pe && !ce) throw Error{HB_ERR_FORMAT, "XML <initialconditions> element contains no known initial condition type"};
  p.initial_density = 1.0;
  if (pe) {
    double p0 = parse_double(dim_value(pe->require("uniform"), "mmHg"), "initial pressure");
    p.initial_density = u.pressure_abs(p0) / kCs2;
  } else {
    c.checkpoint_file = ce->attr("file");
  }
  if (is_sponge(kernel)) {  // SimConfig.cc:707
    const XmlElement& sp = ic.require("sponge_layer");
    p.viscosity_ratio = parse_double(dim_value(sp.require("viscosity_ratio"), "dimensionless"), "viscosity_ratio");
    p.sponge_width = u.to_lattice("m", parse_double(dim_value(sp.require("width"), "m"), "width"));
    p.sponge_lifetime = parse_u64(dim_value(sp.require("lifetime"), "lattice"), "lifetime");
  }

  auto read_iolets = [&](const char* group, hb_iolet* out, int& count, int group_index) {
    const XmlElement& g = root->require(group);
    std::string child = std::string(group).substr(0, std::strlen(group) - 1);
    count = 0;
    for (const XmlElement* el : g.all(child)) {
      if (count >= 16) throw Error{HB_ERR_UNSUPPORTED, std::string("more than 16 ") + group};
      hb_iolet& io = out[count++];
      std::memset(&io, 0, sizeof(io));
      const XmlElement& cond = el->require("condition");
      const std::string& type = cond.attr("type");
      const std::string& sub = cond.attr("subtype");
      parse_vec(dim_value(el->require("position"), "lattice"), io.position, "position");
      parse_vec(dim_value(el->require("normal"), "dimensionless"), io.normal, "normal");
      normalise(io.normal);
      if (type == "pressure" && sub == "cosine") {
        io.kind = kCosine;
        io.density_amp = u.pressure_diff(parse_double(dim_value(cond.require("amplitude"), "mmHg"), "amplitude")) / kCs2;
        io.density_mean = u.pressure_abs(parse_double(dim_value(cond.require("mean"), "mmHg"), "mean")) / kCs2;
        io.phase = u.to_lattice("rad", parse_double(dim_value(cond.require("phase"), "rad"), "phase"));
        io.period = u.to_lattice("s", parse_double(dim_value(cond.require("period"), "s"), "period"));
        io.warmup = c.warmup;
      } else if (type == "pressure" && sub == "WK3") {
        io.kind = kWK3;
        const double rf = (c.dt * c.dx) / kBloodDensity;
        const double cf = kBloodDensity / (c.dt * c.dt * c.dx);
        io.rc = parse_double(dim_value(cond.require("Rc"), "kg/m^4*s"), "Rc") * rf;
        io.rp = parse_double(dim_value(cond.require("Rp"), "kg/m^4*s"), "Rp") * rf;
        io.cp = parse_double(dim_value(cond.require("Cp"), "m^4*s^2/kg"), "Cp") * cf;
        io.radius = u.to_lattice("m", parse_double(dim_value(cond.require("radius"), "m"), "radius"));
        io.area = parse_double(dim_value(cond.require("area"), "m^2"), "area") / (c.dx * c.dx);
      } else if (type == "pressure" && sub == "WK2") {
        io.kind = kWK2;
        io.rp = parse_double(dim_value(cond.require("R"), "kg/m^4*s"), "R") * ((c.dt * c.dx) / kBloodDensity);
        io.cp = parse_double(dim_value(cond.require("C"), "m^4*s^2/kg"), "C") * (kBloodDensity / (c.dt * c.dt * c.dx));
        io.radius = u.to_lattice("m", parse_double(dim_value(cond.require("radius"), "m"), "radius"));
        io.area = parse_double(dim_value(cond.require("area"), "m^2"), "area") / (c.dx * c.dx);
      } else if (type == "pressure" && sub == "file") {
        io.kind = kFile;
        std::string path = cond.require("path").attr("value");
        if (!path.empty() && path[0] != '/') {
          const size_t slash = xml_path.rfind('/');
          if (slash != std::string::npos) path = xml_path.substr(0, slash + 1) + path;
        }
        std::vector<double>& table = c.tables[group_index * 16 + (count - 1)];
        file_density_table(path, c.total_steps, c.dt, u, table, io.density_min);
        io.table = table.data();
        io.table_steps = table.size();
      } else if (type == "pressure" && sub == "fileWK") {
        // InOutLetFileWK: a WK2 whose weights file is read only in builds with
        // HEMELB_USE_VELOCITY_WEIGHTS_FILE, and whose radius is never set.
        io.kind = kWK2;
        cond.require("path");
        io.rp = parse_double(dim_value(cond.require("R"), "kg/m^4*s"), "R") * ((c.dt * c.dx) / kBloodDensity);
        io.cp = parse_double(dim_value(cond.require("C"), "m^4*s^2/kg"), "C") * (kBloodDensity / (c.dt * c.dt * c.dx));
        io.area = parse_double(dim_value(cond.require("area"), "m^2"), "area") / (c.dx * c.dx);
      } else if (type == "velocity" && sub == "file") {
        io.kind = kFileVelocity;
        std::string path = cond.require("path").attr("value");
        if (!path.empty() && path[0] != '/') {
          const size_t slash = xml_path.rfind('/');
          if (slash != std::string::npos) path = xml_path.substr(0, slash + 1) + path;
        }
        io.radius = u.to_lattice("m", parse_double(dim_value(cond.require("radius"), "m"), "radius"));
        std::vector<double>& table = c.tables[group_index * 16 + (count - 1)];
        file_velocity_table(path, c.total_steps, c.dt, u, table);
        io.table = table.data();
        io.table_steps = table.size();
      } else if (type == "velocity" && sub == "womersley") {
        io.kind = kWomersley;
        io.radius = u.to_lattice("m", parse_double(dim_value(cond.require("radius"), "m"), "radius"));
        io.pressure_gradient_amplitude = u.to_lattice(
            "mmHg/m", parse_double(dim_value(cond.require("pressure_gradient_amplitude"), "mmHg/m"), "pressure_gradient_amplitude"));
        io.period = u.to_lattice("s", parse_double(dim_value(cond.require("period"), "s"), "period"));
        io.womersley_number = u.to_lattice(
            "dimensionless", parse_double(dim_value(cond.require("womersley_number"), "dimensionless"), "womersley_number"));
      } else if (type == "velocity" && sub == "parabolic") {
        io.kind = kParabolic;
        io.radius = u.to_lattice("m", parse_double(dim_value(cond.require("radius"), "m"), "radius"));
        io.max_speed = u.to_lattice("m/s", parse_double(dim_value(cond.require("maximum"), "m/s"), "maximum"));
        io.warmup = c.warmup;
      } else {
        throw Error{HB_ERR_UNSUPPORTED, "Invalid boundary condition type/subtype '" + type + "/" + sub + "'"};
      }
    }
  };
  read_iolets("inlets", p.inlets, p.n_inlets, 0);
  read_iolets("outlets", p.outlets, p.n_outlets, 1);

  if (const XmlElement* props = root->child("properties")) {
    for (const XmlElement* po : props->all("propertyoutput")) {
      CaseConfig::PropertyOutput o;
      o.file = po->attr("file");
      o.period = parse_u64(po->attr("period"), "period");
      if (const XmlElement* g = po->child("geometry")) o.geometry = g->attr("type");
      for (const XmlElement* f : po->all("field")) o.fields.push_back(f->attr("type"));
      c.outputs.push_back(o);
    }
  }
  return c;
}

// ---------------------------------------------------------------------------
// Velocity iolets on the host
// ---------------------------------------------------------------------------

// The power series J0(z) = sum_k (-z^2/4)^k / (k!)^2, summed in the order and
// with the stopping rule of util::BesselJ0ComplexArgument: stop once the last
// term's squared modulus is at most tol_sq.
std::complex<double> bessel_j0(const std::complex<double>& z, double tol_sq) {
  std::complex<double> sum(1.0, 0.0), zpow(1.0, 0.0), term(1.0, 0.0);
  double fact = 1;
  for (unsigned k = 1; term.real() * term.real() + term.imag() * term.imag() > tol_sq; ++k) {
    fact *= k;
    zpow *= -0.25 * z * z;
    term = zpow / (fact * fact);
    sum += term;
  }
  return sum;
}

namespace {

// |x - position|^2 - ((x - position) . normal)^2, in the iolets' order of operations
// (InOutLetParabolicVelocity.cc:33-36, InOutLetWomersleyVelocity.cc:28-30).
double radial_sq(const hb_iolet& io, const double x[3]) {
  const double dx = x[0] - io.position[0], dy = x[1] - io.position[1], dz = x[2] - io.position[2];
  const double z = dx * io.normal[0] + dy * io.normal[1] + dz * io.normal[2];
  return (dx * dx + dy * dy + dz * dz) - z * z;
}

}  // namespace

// InOutLetWomersleyVelocity::GetVelocity (src/lb/iolets/InOutLetWomersleyVelocity.cc:25-41)
// without its last factor exp(i omega t); the grouping of the products is the
// reference's, so the host's std::complex arithmetic rounds as it does.
std::complex<double> womersley_amplitude(const hb_iolet& io, const double x[3]) {
  const double r = std::sqrt(radial_sq(io, x));
  const double omega = 2.0 * kPi / io.period;
  const double density = 1.0;
  const std::complex<double> i(0, 1);
  const std::complex<double> i32 = std::pow(i, 1.5);
  const std::complex<double> numer = bessel_j0(i32 * io.womersley_number * r / io.radius);
  const std::complex<double> denom = bessel_j0(i32 * io.womersley_number);
  return io.pressure_gradient_amplitude / (density * omega) * (1.0 - numer / denom);
}

std::complex<double> womersley_phase(const hb_iolet& io, uint64_t t) {
  const std::complex<double> i(0, 1);
  const double omega = 2.0 * kPi / io.period;
  return std::exp(i * omega * double(t));
}

int iolet_velocity(const hb_iolet& io, const double x[3], uint64_t t, double v[3]) {
  if (io.kind == kWomersley) {
    const double speed = std::real(womersley_amplitude(io, x) * womersley_phase(io, t));
    for (int k = 0; k < 3; k++) v[k] = io.normal[k] * -speed;
    return 0;
  }
  if (io.kind != kParabolic && io.kind != kFileVelocity) return HB_ERR_UNSUPPORTED;
  // InOutLetParabolicVelocity::GetVelocity (src/lb/iolets/InOutLetParabolicVelocity.cc:30-58),
  // InOutLetFileVelocity::GetVelocity (src/lb/iolets/InOutLetFileVelocity.cc:104-128).
  const double r2a2 = radial_sq(io, x) / (io.radius * io.radius);
  if (r2a2 > 1.0) return HB_ERR_IOLET_RADIUS;
  double mx;
  if (io.kind == kParabolic) {
    mx = io.max_speed;
    if (t < io.warmup) mx *= (double)t / (double)io.warmup;
  } else {
    if (!io.table || io.table_steps == 0) return HB_ERR_ARG;
    mx = io.table[t < io.table_steps ? t : io.table_steps - 1];
  }
  const double s = mx * (1. - r2a2);
  for (int k = 0; k < 3; k++) v[k] = io.normal[k] * s;
  return 0;
}

// ---------------------------------------------------------------------------
// .gmy reader
// ---------------------------------------------------------------------------

namespace {

struct Xdr {
  const unsigned char* p;
  size_t n, pos = 0;
  bool bad = false;
  uint32_t u32() {
    if (pos + 4 > n) {
      bad = true;
      return 0;
    }
    const unsigned char* b = p + pos;
    pos += 4;
    return (uint32_t(b[0]) << 24) | (uint32_t(b[1]) << 16) | (uint32_t(b[2]) << 8) | uint32_t(b[3]);
  }
  float f32() {
    uint32_t v = u32();
    float f;
    std::memcpy(&f, &v, 4);
    return f;
  }
};

struct ReadSite {
  uint32_t wall = 0, iolet = 0;
  int32_t stype = 0, iolet_id = -1;
  float dist[18];
  bool has_normal = false;
  float normal[3];
};

}  // namespace

void* host_table_alloc(size_t bytes) {
  constexpr size_t kHuge = (size_t)2 << 20;
  if (bytes < 8 * kHuge) {
    void* p = std::malloc(bytes);
    if (!p) throw std::bad_alloc();
    return p;
  }
  const size_t rounded = (bytes + kHuge - 1) / kHuge * kHuge;
  void* p = std::aligned_alloc(kHuge, rounded);
  if (!p) throw std::bad_alloc();
  madvise(p, rounded, MADV_HUGEPAGE);  // advice only: ignored where huge pages are off
  return p;
}

void host_table_free(void* p) { std::free(p); }

LatticeTables read_gmy(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error{HB_ERR_IO, "cannot open geometry file " + path};
  std::vector<unsigned char> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  Xdr x{buf.data(), buf.size()};
  uint32_t hlb = x.u32(), gmy = x.u32(), ver = x.u32();
  if (hlb != 0x686c6221u) throw Error{HB_ERR_FORMAT, "This file does not start with the HemeLB magic number."};
  if (gmy != 0x676d7904u) throw Error{HB_ERR_FORMAT, "This file does not have the geometry magic number."};
  if (ver != 4u) throw Error{HB_ERR_FORMAT, "Version number incorrect."};
  LatticeTables t;
  for (int d = 0; d < 3; d++) t.blocks[d] = x.u32();
  t.block_size = x.u32();
  const int64_t bs = t.block_size, bs3 = bs * bs * bs;
  for (int d = 0; d < 3; d++) t.dims[d] = t.blocks[d] * bs;
  const int64_t nblocks = t.blocks[0] * t.blocks[1] * t.blocks[2];
  if (bs <= 0 || nblocks <= 0) throw Error{HB_ERR_FORMAT, "empty geometry"};
  x.pos = 32;
  std::vector<uint32_t> hdr(3 * nblocks);
  for (int64_t b = 0; b < 3 * nblocks; b++) hdr[b] = x.u32();
  if (x.bad) throw Error{HB_ERR_FORMAT, "truncated header"};

  // Map the 26 .gmy displacements onto D3Q19 directions 1..18.
  int gmy_to_q[26];
  {
    int k = 0;
    for (int dx = -1; dx <= 1; dx++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dz = -1; dz <= 1; dz++) {
          if (!dx && !dy && !dz) continue;
          gmy_to_q[k] = -1;
          for (int d = 1; d < Q; d++)
            if (cx(d) == dx && cy(d) == dy && cz(d) == dz) gmy_to_q[k] = d;
          k++;
        }
  }

  // Decode every non-empty block; remember for each block where its sites went.
  std::vector<ReadSite> sites;
  std::vector<int32_t> local(nblocks * bs3, -1);
  size_t off = 32 + 12 * (size_t)nblocks;
  std::vector<unsigned char> raw;
  for (int64_t b = 0; b < nblocks; b++) {
    if (hdr[3 * b] == 0) continue;
    uint32_t cb = hdr[3 * b + 1], ub = hdr[3 * b + 2];
    if (off + cb > buf.size()) throw Error{HB_ERR_FORMAT, "truncated block data"};
    raw.resize(ub);
    uLongf dl = ub;
    if (uncompress(raw.data(), &dl, buf.data() + off, cb) != Z_OK) throw Error{HB_ERR_FORMAT, "Decompression error for block!"};
    off += cb;
    Xdr bx{raw.data(), (size_t)dl};
    int64_t count = 0;
    for (int64_t s = 0; s < bs3; s++) {
      if (!bx.u32()) continue;
      ReadSite r;
      for (int d = 0; d < 18; d++) r.dist[d] = -1.0f;
      bool gmy_wall = false, had_in = false, had_out = false;
      uint8_t types[18] = {0};
      int32_t ids[18];
      for (int d = 0; d < 18; d++) ids[d] = -1;
      for (int k = 0; k < 26; k++) {
        uint32_t ty = bx.u32();
        float dist = -1.0f;
        int32_t iid = -1;
        if (ty == 1) {
          gmy_wall = true;
          dist = bx.f32();
        } else if (ty != 0) {
          iid = (int32_t)bx.u32();
          dist = bx.f32();
        }
        int d = gmy_to_q[k];
        if (d > 0) {
          types[d - 1] = (uint8_t)ty;
          ids[d - 1] = iid;
          r.dist[d - 1] = dist;
        }
      }
      uint32_t na = bx.u32();
      r.has_normal = (na == 1u);
      if (r.has_normal != gmy_wall)
        throw Error{HB_ERR_FORMAT, std::string("Malformed GMY file, ") + (gmy_wall ? "wall fluid site without" : "bulk fluid site with") +
                                       " a defined wall normal currently not allowed."};
      if (r.has_normal) {
        r.normal[0] = bx.f32();
        r.normal[1] = bx.f32();
        r.normal[2] = bx.f32();
      }
      for (int d = 1; d <= 18; d++) {
        int ty = types[d - 1];
        if (ty == 1) r.wall |= 1u << (d - 1);
        else if (ty == 2 || ty == 3) r.iolet |= 1u << (d - 1);
        if (ty == 2) {
          r.iolet_id = ids[d - 1];
          had_in = true;
        } else if (ty == 3) {
          r.iolet_id = ids[d - 1];
          had_out = true;
        }
      }
      r.stype = had_in ? 1 : (had_out ? 2 : 0);
      local[b * bs3 + s] = (int32_t)sites.size();
      sites.push_back(r);
      count++;
    }
    if (bx.bad) throw Error{HB_ERR_FORMAT, "truncated site record"};
    if (count != (int64_t)hdr[3 * b]) throw Error{HB_ERR_FORMAT, "block fluid-site count does not match its header"};
  }

  // Bin by collision type in block-traversal order (z fastest, then y, then x).
  const int64_t n = (int64_t)sites.size();
  t.n = n;
  auto ctype = [&](const ReadSite& r) {
    const bool w = r.wall != 0;
    return !w ? (r.stype == 0 ? 0 : (r.stype == 1 ? 2 : 3)) : (r.stype == 0 ? 1 : (r.stype == 1 ? 4 : 5));
  };
  for (auto& r : sites) t.type_counts[ctype(r)]++;
  int64_t fill[6];
  fill[0] = 0;
  for (int k = 1; k < 6; k++) fill[k] = fill[k - 1] + t.type_counts[k - 1];
  t.coords.resize(3 * n);
  t.wall.resize(n);
  t.iolet.resize(n);
  t.stype.resize(n);
  t.iolet_id.resize(n);
  t.q.resize(18 * n);
  t.normal.resize(3 * n);
  for (int64_t bxi = 0; bxi < t.blocks[0]; bxi++)
    for (int64_t byi = 0; byi < t.blocks[1]; byi++)
      for (int64_t bzi = 0; bzi < t.blocks[2]; bzi++) {
        const int64_t b = (bxi * t.blocks[1] + byi) * t.blocks[2] + bzi;
        if (hdr[3 * b] == 0) continue;
        for (int64_t s = 0; s < bs3; s++) {
          const int32_t ri = local[b * bs3 + s];
          if (ri < 0) continue;
          const ReadSite& r = sites[ri];
          const int64_t c = fill[ctype(r)]++;
          t.coords[3 * c] = bxi * bs + s / (bs * bs);
          t.coords[3 * c + 1] = byi * bs + (s / bs) % bs;
          t.coords[3 * c + 2] = bzi * bs + s % bs;
          t.wall[c] = r.wall;
          t.iolet[c] = r.iolet;
          t.stype[c] = r.stype;
          t.iolet_id[c] = r.iolet_id;
          for (int d = 0; d < 18; d++) t.q[18 * c + d] = r.dist[d];
          if (r.has_normal) {
            // Vector3D<float>::GetNormalised, in float.
            float nx = r.normal[0], ny = r.normal[1], nz = r.normal[2];
            if (nx == 0.0f && ny == 0.0f && nz == 0.0f) {
              t.normal[3 * c] = t.normal[3 * c + 1] = t.normal[3 * c + 2] = 0.0f;
            } else {
              volatile float m2 = nx * nx + ny * ny + nz * nz;
              float m = std::sqrt((float)m2);
              t.normal[3 * c] = nx / m;
              t.normal[3 * c + 1] = ny / m;
              t.normal[3 * c + 2] = nz / m;
            }
          } else {
            t.normal[3 * c] = t.normal[3 * c + 1] = t.normal[3 * c + 2] = HUGE_VALF;
          }
        }
      }
  return t;
}

void build_neighbours(LatticeTables& t) {
  std::vector<int64_t> nbr((size_t)Q * t.n);
  neighbour_table(t, nbr.data());
  t.nbr = std::move(nbr);
}

void neighbour_table(const LatticeTables& t, int64_t* out) {
  const int64_t n = t.n;
  if (!t.nbr.empty()) {
    std::memcpy(out, t.nbr.data(), (size_t)Q * n * sizeof(int64_t));
    return;
  }
  const int64_t D0 = t.dims[0], D1 = t.dims[1], D2 = t.dims[2];
  std::vector<int32_t> grid(D0 * D1 * D2, -1);
  for (int64_t c = 0; c < n; c++) {
    const int64_t* p = &t.coords[3 * c];
    if (p[0] < 0 || p[1] < 0 || p[2] < 0 || p[0] >= D0 || p[1] >= D1 || p[2] >= D2)
      throw Error{HB_ERR_BAD_INDEX, "site coordinates outside the lattice"};
    int32_t& g = grid[(p[0] * D1 + p[1]) * D2 + p[2]];
    if (g >= 0) throw Error{HB_ERR_BAD_INDEX, "two sites share coordinates"};
    g = (int32_t)c;
  }
  for (int64_t c = 0; c < n; c++) {
    out[Q * c] = Q * c;
    for (int d = 1; d < Q; d++) {
      const int64_t px = t.coords[3 * c] + cx(d), py = t.coords[3 * c + 1] + cy(d), pz = t.coords[3 * c + 2] + cz(d);
      int64_t v = n * Q;  // the rubbish slot
      if (px >= 0 && py >= 0 && pz >= 0 && px < D0 && py < D1 && pz < D2) {
        const int32_t g = grid[(px * D1 + py) * D2 + pz];
        if (g >= 0) v = (int64_t)g * Q + d;
      }
      out[Q * c + d] = v;
    }
  }
}

}  // namespace hb
