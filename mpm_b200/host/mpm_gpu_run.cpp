// mpm_gpu_run -- runs an explicit MPM analysis written in the reference's
// input format on the GPU, through the C ABI of libmpm_b200.so.
//
//   mpm_gpu_run -f <input directory> [-i mpm.json] [--precision fp64|mixed]
//               [--device N] [--parse-only]
//
// The host side of the drop-in: it reads what MPMBase reads for an explicit
// single-phase analysis (mpm_base.tcc:3-207, 347-473, 1550-1625;
// mpm_explicit.tcc:8-13, 62-108) -- the analysis object (scheme,
// velocity_update and blending ratio, dt, nsteps, locate_particles, Cundall
// damping), external loading (gravity, optional ramping time), materials,
// the mesh and particle files (io_mesh_ascii.tcc: mesh, particles,
// particle stresses, velocity and friction constraints), particle entity sets
// (io.cc:159-194) with particle velocity constraints -- and calls the same
// steps on the library.  As MPMBase::write_outputs does (mpm_base.tcc:749-756,
// 577-596; io.cc:94-135) it writes the particles' HDF5 table (the
// PODParticle records of Mesh::write_particles_hdf5, mesh.tcc:1573-1613) to
// <post_processing.path><uuid>/particles<step>.h5 at the first step and
// every output_steps steps, the step zero-padded to the digits of nsteps, and
// prints the solver duration as mpm_explicit.tcc:191-196 does.  With
// analysis.resume.resume true it resumes as MPMBase::checkpoint_resume does
// (mpm_base.tcc:509-551): the particles of particles<resume.step>.h5 of
// resume.uuid, from that step on.
//
// --parse-only reads and checks the input and prints a summary without
// touching a GPU.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "json_lite.hpp"
#include "mpm_gpu.h"

using mpm_b200::Json;

namespace {

struct Input {
  int dim = 3;
  std::string scheme = "usf", vupdate = "flip", uuid = "mpm", out_path = "results/";
  double beta = 1.0, dt = 0.0, damping = 0.0, ramp = 0.0;
  double gravity[3] = {0, 0, 0};
  long nsteps = 0, output_steps = 0;  // output_steps 0: at the start and the end only
  bool resume = false;
  std::string resume_uuid;
  long resume_step = 0;
  bool locate = true;
  bool isoparametric = true;          // mesh "isoparametric" (mpm_base.tcc:767-784 default)
  std::vector<double> coords;         // nnodes x dim
  std::vector<int64_t> cells;         // ncells x nv
  int64_t nnodes = 0, ncells = 0;
  struct Mat {
    int id;
    std::string type, json;
  };
  std::vector<Mat> mats;
  struct PSet {
    std::vector<double> x;            // n x dim
    int material;
  };
  std::vector<PSet> psets;
  std::vector<double> stresses;       // nparticles x 6 (optional)
  std::vector<int64_t> vnid, fnid, enid;
  std::vector<int32_t> vdir, fdir, fsign;
  std::vector<double> vval, fmu, eangles;  // eangles: nodal Euler angles, enid.size() x dim
  struct PVC {
    std::vector<int64_t> ids;         // empty: every particle (set -1)
    int dir;
    double v;
  };
  std::vector<PVC> pvcs;
  struct MatSet {                     // material_sets: every particle of a set takes a material
    int material;
    std::vector<int64_t> ids;
  };
  std::vector<MatSet> matsets;
  std::vector<std::string> unsupported;  // input entries outside the explicit single-phase path
  int64_t nparticles() const {
    int64_t n = 0;
    for (auto& p : psets) n += (int64_t)p.x.size() / dim;
    return n;
  }
};

std::string read_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

// Data lines of a reference ASCII file: comment lines (# or !) and blank
// lines skipped (io_mesh_ascii.tcc:4-140).
std::vector<std::string> data_lines(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::vector<std::string> out;
  std::string line;
  while (std::getline(f, line)) {
    const size_t a = line.find_first_not_of(" \t\r");
    if (a == std::string::npos) continue;
    if (line.find('#') != std::string::npos || line.find('!') != std::string::npos) continue;
    out.push_back(line.substr(a));
  }
  return out;
}

// A reference ASCII data file read whole: the [begin, end) ranges of its data
// lines (the same lines as data_lines keeps).  The large tables (mesh nodes
// and cells, particles, particle stresses) are parsed from it row-parallel.
struct DataFile {
  std::string text;
  std::vector<size_t> begin, end;
  size_t size() const { return begin.size(); }
};

DataFile read_data_file(const std::string& path) {
  DataFile df;
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open " + path);
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  df.text.resize(n > 0 ? (size_t)n : 0);
  const size_t got = n > 0 ? std::fread(&df.text[0], 1, (size_t)n, f) : 0;
  std::fclose(f);
  if (got != df.text.size()) throw std::runtime_error("cannot read " + path);
  const char* t = df.text.data();
  const size_t len = df.text.size();
  size_t pos = 0;
  while (pos < len) {
    const char* nl = static_cast<const char*>(std::memchr(t + pos, '\n', len - pos));
    const size_t e = nl ? (size_t)(nl - t) : len;
    size_t a = pos;
    while (a < e && (t[a] == ' ' || t[a] == '\t' || t[a] == '\r')) ++a;
    if (a < e && !std::memchr(t + pos, '#', e - pos) && !std::memchr(t + pos, '!', e - pos)) {
      df.begin.push_back(a);
      df.end.push_back(e);
    }
    pos = e + 1;
  }
  return df;
}

// Reads up to ncols whitespace-separated numbers of one line into out (values
// left as they are where the line ends early, as operator>> does).
template <typename T>
void parse_line(const DataFile& df, size_t line, int ncols, T* out) {
  const char* p = df.text.data() + df.begin[line];
  const char* e = df.text.data() + df.end[line];
  for (int k = 0; k < ncols; ++k) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    if (p < e && *p == '+') ++p;
    if (p >= e) return;
    const auto r = std::from_chars(p, e, out[k]);
    if (r.ec != std::errc()) return;
    p = r.ptr;
  }
}

// rows [first, first + nrows) of ncols numbers each into out, over all host threads
template <typename T>
void parse_rows(const DataFile& df, size_t first, int64_t nrows, int ncols, T* out) {
  if (first + (size_t)nrows > df.size()) throw std::runtime_error("data file too short");
  const int64_t nt = std::max<int64_t>(
      1, std::min<int64_t>(std::thread::hardware_concurrency(), nrows / 4096 + 1));
  std::vector<std::thread> pool;
  for (int64_t w = 0; w < nt; ++w)
    pool.emplace_back([&, w]() {
      const int64_t a = nrows * w / nt, b = nrows * (w + 1) / nt;
      for (int64_t i = a; i < b; ++i) parse_line(df, first + (size_t)i, ncols, out + i * ncols);
    });
  for (auto& t : pool) t.join();
}

std::string fmt_double(double v) {
  char b[40];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

std::string dump(const Json& j) {
  switch (j.type) {
    case Json::Null: return "null";
    case Json::Bool: return j.b ? "true" : "false";
    case Json::Number: return fmt_double(j.num);
    case Json::String: {
      std::string s = "\"";
      for (char c : j.str) {
        if (c == '"' || c == '\\') s += '\\';
        s += c;
      }
      return s + "\"";
    }
    case Json::Array: {
      std::string s = "[";
      for (size_t i = 0; i < j.arr.size(); ++i) s += (i ? "," : "") + dump(j.arr[i]);
      return s + "]";
    }
    default: {
      std::string s = "{";
      for (size_t i = 0; i < j.obj.size(); ++i)
        s += (i ? ",\"" : "\"") + j.obj[i].first + "\":" + dump(j.obj[i].second);
      return s + "}";
    }
  }
}

std::string join(const std::string& dir, const std::string& f) {
  if (f.empty() || f[0] == '/') return f;
  return dir.empty() || dir.back() == '/' ? dir + f : dir + "/" + f;
}

Input read_input(const std::string& dir, const std::string& file) {
  Input in;
  const Json root = mpm_b200::parse_json(read_file(join(dir, file)));
  const Json& an = root.at("analysis");
  const std::string type = an.at("type").as_string();  // MPMExplicit2D / 3D
  if (type.find("MPMExplicit") != 0) throw std::runtime_error("analysis type " + type + " is not explicit");
  in.dim = type.size() >= 2 && type.substr(type.size() - 2) == "2D" ? 2 : 3;
  in.dt = an.at("dt").as_double();
  in.nsteps = (long)an.at("nsteps").as_double();
  if (an.contains("mpm_scheme")) in.scheme = an.at("mpm_scheme").as_string();
  if (an.contains("velocity_update")) {
    const Json& vu = an.at("velocity_update");
    in.vupdate = vu.is_bool() ? (vu.as_bool() ? "pic" : "flip") : vu.as_string();
  }
  if (an.contains("velocity_update_settings") && an.at("velocity_update_settings").contains("blending_ratio")) {
    in.beta = an.at("velocity_update_settings").at("blending_ratio").as_double();
    if (in.beta < 0. || in.beta > 1.) in.beta = 1.0;  // mpm_base.tcc:89-91
  }
  if (an.contains("locate_particles")) in.locate = an.at("locate_particles").as_bool();
  if (an.contains("damping")) {
    const Json& d = an.at("damping");
    if (d.contains("type") && d.at("type").as_string() == "Cundall") in.damping = d.get("damping_factor", 0.0);
  }
  if (an.contains("uuid")) in.uuid = an.at("uuid").as_string();
  if (root.contains("post_processing") && root.at("post_processing").contains("path"))
    in.out_path = root.at("post_processing").at("path").as_string();
  if (root.contains("post_processing") && root.at("post_processing").contains("output_steps"))
    in.output_steps = (long)root.at("post_processing").at("output_steps").as_double();
  if (root.contains("external_loading_conditions") &&
      root.at("external_loading_conditions").contains("gravity")) {
    const Json& g = root.at("external_loading_conditions").at("gravity");
    const Json& gv = g.is_array() ? g : g.at("gravity");
    if (!g.is_array() && g.contains("ramping_time")) in.ramp = g.at("ramping_time").as_double();
    if ((int)gv.size() != in.dim) throw std::runtime_error("gravity dimension is invalid");
    for (int d = 0; d < in.dim; ++d) in.gravity[d] = gv.at(d).as_double();
  }
  for (const Json& m : root.at("materials").arr)
    in.mats.push_back({(int)m.at("id").as_double(), m.at("type").as_string(), dump(m)});
  // mesh (io_mesh_ascii.tcc: "nnodes ncells", node coordinates, cell node ids)
  const Json& mesh = root.at("mesh");
  if (mesh.contains("isoparametric")) in.isoparametric = mesh.at("isoparametric").as_bool();
  {
    const DataFile df = read_data_file(join(dir, mesh.at("mesh").as_string()));
    if (df.size() == 0) throw std::runtime_error("empty mesh file");
    int64_t hdr[2] = {0, 0};
    parse_line(df, 0, 2, hdr);
    in.nnodes = hdr[0];
    in.ncells = hdr[1];
    const int nv = in.dim == 2 ? 4 : 8;
    if ((int64_t)df.size() < 1 + in.nnodes + in.ncells) throw std::runtime_error("mesh file too short");
    in.coords.assign((size_t)in.nnodes * in.dim, 0.);
    parse_rows(df, 1, in.nnodes, in.dim, in.coords.data());
    in.cells.assign((size_t)in.ncells * nv, 0);
    parse_rows(df, 1 + (size_t)in.nnodes, in.ncells, nv, in.cells.data());
  }
  // particles (a count, then coordinates), one file per generator
  for (const Json& p : root.at("particles").arr) {
    const Json& g = p.at("generator");
    if (g.at("type").as_string() != "file") throw std::runtime_error("particle generator must be a file");
    const DataFile df = read_data_file(join(dir, g.at("location").as_string()));
    if (df.size() == 0) throw std::runtime_error("empty particle file");
    Input::PSet ps;
    ps.material = (int)g.at("material_id").as_double();
    int64_t n = 0;
    parse_line(df, 0, 1, &n);
    ps.x.assign((size_t)n * in.dim, 0.);
    parse_rows(df, 1, n, in.dim, ps.x.data());
    in.psets.push_back(std::move(ps));
  }
  if (mesh.contains("particles_stresses")) {
    const Json& ps = mesh.at("particles_stresses");
    if (ps.at("type").as_string() != "file") throw std::runtime_error("only file particle stresses are read");
    const DataFile df = read_data_file(join(dir, ps.at("location").as_string()));
    if (df.size() == 0) throw std::runtime_error("empty particle stress file");
    int64_t n = 0;
    parse_line(df, 0, 1, &n);
    in.stresses.assign((size_t)n * 6, 0.);
    parse_rows(df, 1, n, 6, in.stresses.data());
  }
  // particle entity sets (mpm_base.tcc:1731-1760, io.cc:159-194): id -> particle ids
  std::map<long, std::vector<int64_t>> sets;
  if (mesh.contains("entity_sets")) {
    const Json es = mpm_b200::parse_json(read_file(join(dir, mesh.at("entity_sets").as_string())));
    if (es.contains("particle_sets"))
      for (const Json& s : es.at("particle_sets").arr) {
        std::vector<int64_t> ids;
        for (const Json& i : s.at("set").arr) ids.push_back((int64_t)i.as_double());
        sets[(long)s.at("id").as_double()] = ids;
      }
  }
  // material sets (mpm_base.tcc:448-472): applied before the mass is computed
  if (root.contains("material_sets") && root.at("material_sets").is_array())
    for (const Json& m : root.at("material_sets").arr) {
      if (m.contains("phase_id") && (int)m.at("phase_id").as_double() != 0)
        throw std::runtime_error("material_sets: only the solid phase (phase_id 0) exists here");
      const long set = (long)m.at("pset_id").as_double();
      auto it = sets.find(set);
      if (it == sets.end()) throw std::runtime_error("material_sets: unknown particle set " + std::to_string(set));
      in.matsets.push_back({(int)m.at("material_id").as_double(), it->second});
    }
  // entries the reference would act on but this explicit single-phase path
  // does not build: a run refuses them rather than silently dropping a load
  if (root.contains("external_loading_conditions")) {
    const Json& el = root.at("external_loading_conditions");
    for (const char* k : {"particle_surface_traction", "concentrated_nodal_forces", "rotation_forces"})
      if (el.contains(k) && !(el.at(k).is_array() && el.at(k).arr.empty()))
        in.unsupported.push_back(std::string("external_loading_conditions.") + k);
  }
  if (an.contains("resume") && an.at("resume").contains("resume")) {
    const Json& r = an.at("resume");
    const Json& on = r.at("resume");
    // a string "true" is not a JSON bool: the reference's get<bool>() throws and
    // the analysis restarts (mpm_base.tcc:520, 544-548)
    in.resume = on.is_bool() && on.as_bool();
    if (in.resume) {
      in.resume_uuid = r.contains("uuid") ? r.at("uuid").as_string() : in.uuid;
      in.resume_step = r.contains("step") ? (long)r.at("step").as_double() : 0;
    }
  }
  for (const char* k : {"pressure_smoothing", "interface", "pore_pressure_smoothing"})
    if (an.contains(k) && an.at(k).is_bool() && an.at(k).as_bool())
      in.unsupported.push_back(std::string("analysis.") + k);
  if (mesh.contains("boundary_conditions")) {
    const Json& bc = mesh.at("boundary_conditions");
    for (const auto& kv : bc.obj) {
      const std::string& k = kv.first;
      if (k != "velocity_constraints" && k != "friction_constraints" && k != "nodal_euler_angles" &&
          k != "particles_velocity_constraints")
        in.unsupported.push_back("mesh.boundary_conditions." + k);
    }
    // a constraint entry that is not a list of objects makes the reference's
    // reader throw inside its try block and apply none (mpm_base.tcc:1128-1170,
    // 1236-1270): warn and apply none as well
    for (const char* k : {"velocity_constraints", "friction_constraints"})
      if (bc.contains(k) && !bc.at(k).is_array())
        std::fprintf(stderr, "mpm_gpu_run: warning: boundary_conditions.%s is not a list; none applied\n", k);
    if (bc.contains("velocity_constraints"))
      for (const Json& v : bc.at("velocity_constraints").arr)
        for (const auto& line : data_lines(join(dir, v.at("file").as_string()))) {
          std::istringstream l(line);
          int64_t n;
          int d;
          double val;
          l >> n >> d >> val;
          in.vnid.push_back(n);
          in.vdir.push_back(d);
          in.vval.push_back(val);
        }
    if (bc.contains("friction_constraints"))
      for (const Json& v : bc.at("friction_constraints").arr)
        for (const auto& line : data_lines(join(dir, v.at("file").as_string()))) {
          std::istringstream l(line);
          int64_t n;
          int d, sgn;
          double mu;
          l >> n >> d >> sgn >> mu;
          in.fnid.push_back(n);
          in.fdir.push_back(d);
          in.fsign.push_back(sgn);
          in.fmu.push_back(mu);
        }
    // mpm_base.tcc:1041-1063, io_mesh_ascii.tcc:351-390: "nid a0 a1 (a2)" per line
    if (bc.contains("nodal_euler_angles"))
      for (const auto& line : data_lines(join(dir, bc.at("nodal_euler_angles").as_string()))) {
        std::istringstream l(line);
        int64_t n;
        l >> n;
        in.enid.push_back(n);
        for (int d = 0; d < in.dim; ++d) {
          double a = 0.;
          l >> a;
          in.eangles.push_back(a);
        }
      }
    if (bc.contains("particles_velocity_constraints")) {
      for (const Json& c : bc.at("particles_velocity_constraints").arr) {
        const long set = (long)c.at("pset_id").as_double();
        Input::PVC p;
        p.dir = (int)c.at("dir").as_double();
        p.v = c.at("velocity").as_double();
        if (set != -1) {
          auto it = sets.find(set);
          if (it == sets.end()) throw std::runtime_error("unknown particle set " + std::to_string(set));
          p.ids = it->second;
        }
        in.pvcs.push_back(std::move(p));
      }
    }
  }
  return in;
}

// io.cc:94-135: <path><uuid>/<attribute><step, zero-padded to the digits of
// max_steps><extension>
std::string output_file(const std::string& dir, const Input& in, const std::string& uuid, long step) {
  const int digits = (int)std::log10((double)std::max(in.nsteps, 1L)) + 1;
  char num[32];
  std::snprintf(num, sizeof(num), "%0*ld", digits, step);
  const std::string folder = join(join(dir, in.out_path), uuid) + "/";
  return folder + "particles" + num + ".h5";
}

int check(mpm_gpu_t h, int rc, const char* what) {
  if (rc != MPM_OK) {
    std::fprintf(stderr, "mpm_gpu_run: %s failed (%d): %s\n", what, rc, h ? mpm_gpu_last_error(h) : "");
    std::exit(1);
  }
  return rc;
}

}  // namespace

int main(int argc, char** argv) {
  std::string dir, file = "mpm.json", precision = "fp64";
  int device = 0;
  bool parse_only = false;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "-f" && i + 1 < argc) dir = argv[++i];
    else if (a == "-i" && i + 1 < argc) file = argv[++i];
    else if (a == "--precision" && i + 1 < argc) precision = argv[++i];
    else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (a == "--parse-only") parse_only = true;
    else {
      std::fprintf(stderr, "usage: mpm_gpu_run -f <dir> [-i mpm.json] [--precision fp64|mixed] "
                           "[--device N] [--parse-only]\n");
      return 2;
    }
  }
  Input in;
  try {
    in = read_input(dir, file);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "mpm_gpu_run: %s\n", e.what());
    return 1;
  }
  const int64_t np = in.nparticles();
  std::printf("dim %d nodes %lld cells %lld particles %lld materials %zu scheme %s velocity_update %s "
              "dt %g nsteps %ld velocity_constraints %zu friction_constraints %zu "
              "particle_velocity_constraints %zu stresses %s material_sets %zu\n",
              in.dim, (long long)in.nnodes, (long long)in.ncells, (long long)np, in.mats.size(),
              in.scheme.c_str(), in.vupdate.c_str(), in.dt, in.nsteps, in.vnid.size(), in.fnid.size(),
              in.pvcs.size(), in.stresses.empty() ? "no" : "yes", in.matsets.size());
  for (const auto& u : in.unsupported) std::printf("unsupported %s\n", u.c_str());
  if (parse_only) return 0;
  if (!in.unsupported.empty()) {
    std::fprintf(stderr, "mpm_gpu_run: unsupported input: %s%s\n", in.unsupported[0].c_str(),
                 in.unsupported.size() > 1 ? " (and more, see --parse-only)" : "");
    return 1;
  }

  mpm_gpu_config cfg{};
  cfg.dim = in.dim;
  cfg.scheme = in.scheme == "usl" ? MPM_SCHEME_USL : (in.scheme == "musl" ? MPM_SCHEME_MUSL : MPM_SCHEME_USF);
  // mpm_base.tcc: velocity_update "flip", "pic", "asflip", "tpic", "apic"
  if (in.vupdate == "pic")
    cfg.velocity_update = MPM_VELOCITY_PIC;
  else if (in.vupdate == "asflip")
    cfg.velocity_update = MPM_VELOCITY_ASFLIP;
  else if (in.vupdate == "tpic")
    cfg.velocity_update = MPM_VELOCITY_TPIC;
  else if (in.vupdate == "apic")
    cfg.velocity_update = MPM_VELOCITY_APIC;
  else
    cfg.velocity_update = MPM_VELOCITY_FLIP;
  cfg.precision = precision == "mixed" ? MPM_PRECISION_MIXED : MPM_PRECISION_FP64;
  cfg.blending_ratio = in.beta;
  cfg.dt = in.dt;
  cfg.damping_factor = in.damping;
  for (int d = 0; d < 3; ++d) cfg.gravity[d] = in.gravity[d];
  cfg.gravity_ramping_time = in.ramp;
  cfg.locate_particles = in.locate ? 1 : 0;
  cfg.device = device;
  mpm_gpu_t h = nullptr;
  check(nullptr, mpm_gpu_create(&cfg, &h), "create");
  check(h, mpm_gpu_set_mesh(h, in.nnodes, in.coords.data(), in.ncells, in.dim == 2 ? 4 : 8,
                            in.cells.data()), "set_mesh");
  check(h, mpm_gpu_set_isoparametric(h, in.isoparametric ? 1 : 0), "set_isoparametric");
  for (auto& m : in.mats) check(h, mpm_gpu_add_material(h, m.id, m.type.c_str(), m.json.c_str()), "add_material");
  if (!in.vnid.empty())
    check(h, mpm_gpu_add_velocity_constraints(h, (int64_t)in.vnid.size(), in.vnid.data(), in.vdir.data(),
                                              in.vval.data()), "velocity constraints");
  if (!in.fnid.empty())
    check(h, mpm_gpu_add_friction_constraints(h, (int64_t)in.fnid.size(), in.fnid.data(), in.fdir.data(),
                                              in.fsign.data(), in.fmu.data()), "friction constraints");
  if (!in.enid.empty())
    check(h, mpm_gpu_set_nodal_euler_angles(h, (int64_t)in.enid.size(), in.enid.data(),
                                            in.eangles.data()), "nodal Euler angles");
  for (auto& p : in.psets)
    check(h, mpm_gpu_add_particles(h, (int64_t)p.x.size() / in.dim, p.x.data(), p.material), "add_particles");
  for (auto& m : in.matsets)
    check(h, mpm_gpu_assign_particle_materials(h, (int64_t)m.ids.size(), m.ids.data(), m.material),
          "material sets");
  long step0 = 0;
  if (in.resume) {
    // mesh and materials as usual, the particles from the checkpoint file
    const std::string f = output_file(dir, in, in.resume_uuid, in.resume_step);
    if (mpm_gpu_load_hdf5(h, f.c_str()) != MPM_OK) {
      std::fprintf(stderr, "mpm_gpu_run: resume from %s failed: %s; restarting the analysis\n", f.c_str(),
                   mpm_gpu_last_error(h));
      in.resume = false;
    } else {
      step0 = in.resume_step;
      in.uuid = in.resume_uuid;
      check(h, mpm_gpu_set_current_step(h, step0), "set_current_step");
      std::printf("Checkpoint resume at step %ld of %ld\n", step0, in.nsteps);
    }
  }
  if (!in.resume) {
    for (auto& m : in.matsets)
      check(h, mpm_gpu_assign_particle_materials(h, (int64_t)m.ids.size(), m.ids.data(), m.material),
            "material sets");
    check(h, mpm_gpu_initialise(h), "initialise");
    if (!in.stresses.empty())
      check(h, mpm_gpu_assign_particle_stresses(h, (int64_t)in.stresses.size() / 6, in.stresses.data()),
            "particle stresses");
  }
  for (auto& c : in.pvcs)
    check(h, mpm_gpu_add_particle_velocity_constraint(h, c.ids.empty() ? -1 : (int64_t)c.ids.size(),
                                                      c.ids.data(), c.dir, c.v), "particle velocity constraint");
  auto write = [&](long step) {
    const std::string f = output_file(dir, in, in.uuid, step);
    const std::string folder = f.substr(0, f.rfind('/'));
    const std::string cmd = "mkdir -p '" + folder + "'";
    if (std::system(cmd.c_str()) != 0) std::fprintf(stderr, "mpm_gpu_run: cannot create %s\n", folder.c_str());
    check(h, mpm_gpu_write_hdf5(h, f.c_str()), "write_hdf5");
    std::printf("wrote %s\n", f.c_str());
  };
  // mpm_explicit.tcc:108, 189: outputs at the start (not on resume) and after
  // every step that completes a multiple of output_steps
  const long every = in.output_steps > 0 ? in.output_steps : std::max(in.nsteps, 1L);
  if (!in.resume) write(0);
  double total_ms = 0.0;
  for (long s = step0; s < in.nsteps;) {
    const long next = std::min(in.nsteps, (s / every + 1) * every);
    double ms = 0.0;
    check(h, mpm_gpu_step_timed(h, next - s, &ms), "step");
    total_ms += ms;
    s = next;
    if (s % every == 0) write(s);
  }
  std::printf("Explicit solver duration: %.3f ms\n", total_ms);
  mpm_gpu_destroy(h);
  return 0;
}
