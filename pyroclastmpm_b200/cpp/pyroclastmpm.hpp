// Drop-in C++ classes with the reference's names and interfaces (one
// dimension per build, -DDIM=2 or 3, as the reference builds MPM2D / MPM3D).
// They are host views over the C ABI in pmpm.h: containers hold host arrays
// until a solver binds them, after which their fields read and write the
// device state of the solver's simulation handle.
//
//   set_globals            src/common/global_settings.cpp:161-176
//   NodesContainer         include/pyroclastmpm/nodes/nodes.h:73-144
//   ParticlesContainer     include/pyroclastmpm/particles/particles.h:94-271
//   LinearElastic, NewtonFluid, Material    include/pyroclastmpm/materials/*.h
//   Gravity, NodeDomain, BodyForce, PlanarDomain  include/pyroclastmpm/boundaryconditions/*.h
//   Solver, USL            include/pyroclastmpm/solver/{solver.h,usl/usl.h}
//
// Vectors are std::array (the reference uses Eigen fixed-size matrices).
#pragma once

#include <array>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <variant>
#include <vector>

#include "pmpm.h"

#ifndef DIM
#define DIM 3
#endif

namespace pyroclastmpm {
// the 2D and 3D builds are distinct C++ types (both modules may be loaded in
// one process), as the reference's per-DIM libraries are
#if DIM == 2
inline namespace dim2 {
#else
inline namespace dim3 {
#endif

using Real = float;
using Vectorr = std::array<Real, DIM>;
using Vectori = std::array<int, DIM>;
using Matrixr = std::array<Real, DIM * DIM>;
using Matrix3r = std::array<Real, 9>;

inline void check(int status, const char *what) {
  if (status != PMPM_OK) throw std::runtime_error(std::string(what) + ": " + pmpm_status_string(status));
}

// ---------------------------------------------------------------------------
// globals (per process, read when a solver is constructed, as the reference)
// ---------------------------------------------------------------------------
struct Globals {
  Real dt = 0.0f;
  int particles_per_cell = 1;
  int shape_function = PMPM_SHAPE_LINEAR;
  int step = 0;
  std::string output_directory = "./output/";
};
inline Globals &globals() {
  static Globals g;
  return g;
}
inline int shape_function_id(const std::string &name) {
  if (name == "linear") return PMPM_SHAPE_LINEAR;
  if (name == "quadratic") return PMPM_SHAPE_QUADRATIC;
  if (name == "cubic") return PMPM_SHAPE_CUBIC;
  throw std::invalid_argument("shape function must be \"linear\", \"quadratic\" or \"cubic\"");
}
inline void set_global_shapefunction(const std::string &name) { globals().shape_function = shape_function_id(name); }
inline void set_global_timestep(Real dt) { globals().dt = dt; }
inline void set_global_step(int step) { globals().step = step; }
inline void set_global_particles_per_cell(int ppc) { globals().particles_per_cell = ppc; }
inline void set_global_output_directory(const std::string &dir) { globals().output_directory = dir; }
inline void set_globals(Real dt, int ppc, const std::string &shape, const std::string &dir) {
  set_global_timestep(dt);
  set_global_shapefunction(shape);
  set_global_output_directory(dir);
  set_global_particles_per_cell(ppc);
}

// ---------------------------------------------------------------------------
// output (write_vtk_polydata, src/common/output.cpp:132-191): point sets with
// named point arrays, written without VTK: "vtk" -> <stem><step>.vtp (XML
// PolyData, ASCII), "csv" -> <stem><step>.csv (one column per component,
// "Name:k", as vtkDelimitedTextWriter), "obj" -> <stem><step>.obj (vertices)
// ---------------------------------------------------------------------------
struct OutputArray {
  std::string name;
  int ncomp;
  std::vector<double> data;  // [n][ncomp]
};

inline void write_point_set(const std::string &directory, const std::string &stem, int step, double time,
                            const std::vector<double> &points3, const std::vector<OutputArray> &arrays,
                            const std::vector<std::string> &formats) {
  const size_t n = points3.size() / 3;
  std::string base = directory;
  if (!base.empty() && base.back() != '/') base += "/";
  base += stem + std::to_string(step);
  for (const std::string &fmt : formats) {
    std::ostringstream o;
    o << std::setprecision(9);
    if (fmt == "vtk") {
      o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"PolyData\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
        << "<PolyData>\n<FieldData>\n<DataArray type=\"Float64\" Name=\"Time\" NumberOfTuples=\"1\" "
        << "format=\"ascii\">" << time << "</DataArray>\n</FieldData>\n"
        << "<Piece NumberOfPoints=\"" << n << "\" NumberOfVerts=\"0\" NumberOfLines=\"0\" NumberOfStrips=\"0\" "
        << "NumberOfPolys=\"0\">\n<PointData>\n";
      for (const OutputArray &a : arrays) {
        o << "<DataArray type=\"Float64\" Name=\"" << a.name << "\" NumberOfComponents=\"" << a.ncomp
          << "\" format=\"ascii\">\n";
        for (double v : a.data) o << v << " ";
        o << "\n</DataArray>\n";
      }
      o << "</PointData>\n<Points>\n<DataArray type=\"Float32\" Name=\"Points\" NumberOfComponents=\"3\" "
        << "format=\"ascii\">\n";
      for (double v : points3) o << v << " ";
      o << "\n</DataArray>\n</Points>\n</Piece>\n</PolyData>\n</VTKFile>\n";
    } else if (fmt == "csv") {
      bool first = true;
      for (const OutputArray &a : arrays)
        for (int k = 0; k < a.ncomp; k++) {
          o << (first ? "" : ",") << "\"" << a.name << (a.ncomp > 1 ? ":" + std::to_string(k) : "") << "\"";
          first = false;
        }
      o << "\n";
      for (size_t i = 0; i < n; i++) {
        first = true;
        for (const OutputArray &a : arrays)
          for (int k = 0; k < a.ncomp; k++) {
            o << (first ? "" : ",") << a.data[i * a.ncomp + k];
            first = false;
          }
        o << "\n";
      }
    } else if (fmt == "obj") {
      for (size_t i = 0; i < n; i++) o << "v " << points3[3 * i] << " " << points3[3 * i + 1] << " " << points3[3 * i + 2] << "\n";
    } else {
      throw std::invalid_argument("output format must be \"vtk\", \"csv\" or \"obj\" (no glTF writer here)");
    }
    const std::string ext = fmt == "vtk" ? ".vtp" : "." + fmt;
    std::ofstream f(base + ext);
    if (!f) throw std::runtime_error("cannot write " + base + ext);
    f << o.str();
  }
}

// the simulation handle shared by a solver and the containers bound to it
struct SimHandle {
  pmpm_sim *sim = nullptr;
  ~SimHandle() {
    if (sim) pmpm_destroy(sim);
  }
};

// ---------------------------------------------------------------------------
// nodes
// ---------------------------------------------------------------------------
class NodesContainer {
 public:
  NodesContainer() = default;
  NodesContainer(const Vectorr &origin, const Vectorr &end, Real cell_size)
      : origin(origin), end(end), cell_size(cell_size) {
    // Grid ctor (include/pyroclastmpm/common/types_common.h:260-272)
    num_cells_total = 1;
    for (int a = 0; a < DIM; a++) {
      num_cells[a] = (int)((end[a] - origin[a]) / cell_size) + 1;
      num_cells_total *= num_cells[a];
    }
  }
  Vectorr origin{}, end{};
  Real cell_size = 1.0f;
  Vectori num_cells{};
  int num_cells_total = 0;
  std::shared_ptr<SimHandle> handle;

  std::vector<Real> field(int id, int ncomp) const {
    std::vector<Real> out((size_t)num_cells_total * ncomp, 0.0f);
    if (handle) check(pmpm_get_field(handle->sim, id, out.data(), out.size() * sizeof(Real), 0), "nodes field");
    return out;
  }
  std::vector<std::string> output_formats;
  // NodesContainer::output_vtk (src/nodes/nodes.cpp:215-250): the reference
  // writes nodes only while the global step is at most 1
  void output_vtk(int step, double time, const std::string &directory) const {
    if (output_formats.empty() || step > 1) return;
    const std::vector<Real> xyz = give_coords();
    std::vector<double> pts((size_t)num_cells_total * 3, 0.0);
    for (int i = 0; i < num_cells_total; i++)
      for (int a = 0; a < DIM; a++) pts[(size_t)i * 3 + a] = xyz[(size_t)i * DIM + a];
    auto arr = [](const std::string &name, int nc, const std::vector<Real> &v) {
      return OutputArray{name, nc, std::vector<double>(v.begin(), v.end())};
    };
    write_point_set(directory, "nodes", step, time, pts,
                    {arr("Moments", DIM, moments()), arr("MomentsNT", DIM, moments_nt()), arr("Mass", 1, masses())},
                    output_formats);
  }
  std::vector<Real> masses() const { return field(PMPM_FIELD_NODE_MASSES, 1); }
  std::vector<Real> moments() const { return field(PMPM_FIELD_NODE_MOMENTS, DIM); }
  std::vector<Real> moments_nt() const { return field(PMPM_FIELD_NODE_MOMENTS_NT, DIM); }
  // give_node_coords (src/nodes/nodes.cpp:190-205): x-fastest
  std::vector<Real> give_coords() const {
    std::vector<Real> out((size_t)num_cells_total * DIM);
    for (int i = 0; i < num_cells_total; i++) {
      int rem = i;
      for (int a = 0; a < DIM; a++) {
        const int id = rem % num_cells[a];
        rem /= num_cells[a];
        out[(size_t)i * DIM + a] = origin[a] + (Real)id * cell_size;
      }
    }
    return out;
  }
};

// ---------------------------------------------------------------------------
// particles
// ---------------------------------------------------------------------------
class ParticlesContainer {
 public:
  ParticlesContainer() = default;
  ParticlesContainer(const std::vector<Real> &positions, const std::vector<Real> &velocities,
                     const std::vector<int> &colors, const std::vector<Real> &rigid_positions,
                     const std::vector<Real> &rigid_velocities, const std::vector<int> &rigid_colors)
      : positions_(positions), velocities_(velocities), rigid_positions_(rigid_positions),
        rigid_velocities_(rigid_velocities) {
    for (int c : colors) colors_.push_back((unsigned char)c);
    for (int c : rigid_colors) rigid_colors_.push_back((unsigned char)c);
    num_particles = (int)((positions.size() + rigid_positions.size()) / DIM);
  }
  int num_particles = 0;
  std::shared_ptr<SimHandle> handle;
  // host values set before a solver exists (applied when it binds)
  std::vector<std::pair<int, std::vector<unsigned char>>> pending;

  std::vector<Real> positions_, velocities_, rigid_positions_, rigid_velocities_;
  std::vector<unsigned char> colors_, rigid_colors_;

  template <typename T>
  std::vector<T> get(int id, size_t ncomp) const {
    std::vector<T> out((size_t)num_particles * ncomp);
    if (!handle) throw std::runtime_error("the container is not bound to a solver yet");
    check(pmpm_get_field(handle->sim, id, out.data(), out.size() * sizeof(T), 0), "particles field");
    return out;
  }
  template <typename T>
  void set(int id, const std::vector<T> &v, size_t ncomp) {
    if (v.size() != (size_t)num_particles * ncomp) throw std::invalid_argument("wrong number of values");
    if (!handle) {
      std::vector<unsigned char> raw((const unsigned char *)v.data(), (const unsigned char *)(v.data() + v.size()));
      pending.emplace_back(id, raw);
      return;
    }
    check(pmpm_set_field(handle->sim, id, v.data(), v.size() * sizeof(T), 0), "particles field");
  }
  void apply_pending() {
    for (auto &kv : pending) check(pmpm_set_field(handle->sim, kv.first, kv.second.data(), kv.second.size(), 0), "set");
    pending.clear();
  }

  std::vector<std::string> output_formats;
  bool exclude_rigid_from_output = true;
  // ParticlesContainer::output_vtk (src/particles/particles.cpp:209-318): the
  // state plus pressure p = tr(sigma_DIM)/3, q = sqrt(3/2 s:s), |q|/p as
  // |q|/(-p), volumetric strain -tr(eps) and deviatoric strain
  // sqrt(1/2 e:e) of eps = (F + F^T)/2 - I; rigid particles left out
  void output_vtk(int step, double time, const std::string &directory) const {
    if (output_formats.empty() || !handle) return;
    const size_t n = (size_t)num_particles;
    const auto x = get<Real>(PMPM_FIELD_POSITIONS, DIM), v = get<Real>(PMPM_FIELD_VELOCITIES, DIM);
    const auto S = get<Real>(PMPM_FIELD_STRESSES, 9), L = get<Real>(PMPM_FIELD_VELOCITY_GRADIENT, DIM * DIM);
    const auto F = get<Real>(PMPM_FIELD_F, DIM * DIM), m = get<Real>(PMPM_FIELD_MASSES, 1);
    const auto V = get<Real>(PMPM_FIELD_VOLUMES, 1), V0 = get<Real>(PMPM_FIELD_VOLUMES_ORIGINAL, 1);
    const auto col = get<unsigned char>(PMPM_FIELD_COLORS, 1), rig = get<unsigned char>(PMPM_FIELD_IS_RIGID, 1);
    std::vector<size_t> keep;
    for (size_t i = 0; i < n; i++)
      if (!(exclude_rigid_from_output && rig[i])) keep.push_back(i);
    std::vector<double> pts(keep.size() * 3, 0.0);
    std::vector<OutputArray> arrays;
    auto add = [&](const std::string &name, int nc, auto &&value) {
      OutputArray a{name, nc, std::vector<double>(keep.size() * nc)};
      for (size_t j = 0; j < keep.size(); j++)
        for (int k = 0; k < nc; k++) a.data[j * nc + k] = value(keep[j], k);
      arrays.push_back(std::move(a));
    };
    for (size_t j = 0; j < keep.size(); j++)
      for (int a = 0; a < DIM; a++) pts[j * 3 + a] = x[keep[j] * DIM + a];
    std::vector<double> p(n), q(n), mu(n), dev(n), vol(n);
    for (size_t i = 0; i < n; i++) {
      const Real *s = &S[i * 9];
      double tr = 0.0;
      for (int a = 0; a < DIM; a++) tr += s[4 * a];
      p[i] = tr / 3.0;
      double ss = 0.0;
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          const double d = s[3 * a + b] - (a == b ? p[i] : 0.0);
          ss += d * d;
        }
      q[i] = std::sqrt(1.5 * ss);
      mu[i] = std::fabs(q[i]) / (-p[i]);
      double e[DIM * DIM], etr = 0.0;
      for (int a = 0; a < DIM; a++)
        for (int b = 0; b < DIM; b++) {
          e[a * DIM + b] = 0.5 * (F[i * DIM * DIM + a * DIM + b] + F[i * DIM * DIM + b * DIM + a]) - (a == b ? 1.0 : 0.0);
          if (a == b) etr += e[a * DIM + b];
        }
      vol[i] = -etr;
      double es = 0.0;
      for (int a = 0; a < DIM; a++)
        for (int b = 0; b < DIM; b++) {
          const double d = e[a * DIM + b] + (a == b ? vol[i] / 3.0 : 0.0);
          es += d * d;
        }
      dev[i] = std::sqrt(0.5 * es);
    }
    add("isRigid", 1, [&](size_t i, int) { return (double)rig[i]; });
    add("Positions", DIM, [&](size_t i, int k) { return (double)x[i * DIM + k]; });
    add("Velocity", DIM, [&](size_t i, int k) { return (double)v[i * DIM + k]; });
    add("Stress", 9, [&](size_t i, int k) { return (double)S[i * 9 + k]; });
    add("VelocityGradient", DIM * DIM, [&](size_t i, int k) { return (double)L[i * DIM * DIM + k]; });
    add("DeformationMatrix", DIM * DIM, [&](size_t i, int k) { return (double)F[i * DIM * DIM + k]; });
    add("Mass", 1, [&](size_t i, int) { return (double)m[i]; });
    add("Volume", 1, [&](size_t i, int) { return (double)V[i]; });
    add("VolumeOriginal", 1, [&](size_t i, int) { return (double)V0[i]; });
    add("Color", 1, [&](size_t i, int) { return (double)col[i]; });
    add("Pressure", 1, [&](size_t i, int) { return p[i]; });
    add("q", 1, [&](size_t i, int) { return q[i]; });
    add("|q|/p", 1, [&](size_t i, int) { return mu[i]; });
    add("dev strain", 1, [&](size_t i, int) { return dev[i]; });
    add("vol strain", 1, [&](size_t i, int) { return vol[i]; });
    write_point_set(directory, "particles", step, time, pts, arrays, output_formats);
  }
};

// ---------------------------------------------------------------------------
// materials and boundary conditions
// ---------------------------------------------------------------------------
struct Material {
  Real density = 0.0f;
  pmpm_material desc() const {
    pmpm_material m{};
    m.type = PMPM_MAT_NONE;
    m.density = density;
    return m;
  }
};
struct LinearElastic {
  LinearElastic(Real density, Real E, Real pois) : density(density), E(E), pois(pois) {
    // LinearElastic::LinearElastic (src/materials/linearelastic.cpp:47-58)
    bulk_modulus = E / (3.0f * (1.0f - 2.0f * pois));
    shear_modulus = E / (2.0f * (1.0f + pois));
    lame_modulus = E * pois / ((1.0f + pois) * (1.0f - 2.0f * pois));
  }
  Real density, E, pois, bulk_modulus, shear_modulus, lame_modulus;
  bool corrected = false;
  pmpm_material desc() const {
    pmpm_material m;
    check(pmpm_material_linear_elastic(density, E, pois, corrected ? 1 : 0, &m), "LinearElastic");
    return m;
  }
  // LinearElastic::calculate_timestep (src/materials/linearelastic.cpp:96-105)
  Real calculate_timestep(Real cell_size, Real factor) const {
    Real dt;
    check(pmpm_calculate_timestep(cell_size, factor, bulk_modulus, shear_modulus, density, &dt),
          "calculate_timestep");
    return dt;
  }
};
struct NewtonFluid {
  NewtonFluid(Real density, Real viscosity, Real bulk_modulus, Real gamma)
      : density(density), viscosity(viscosity), bulk_modulus(bulk_modulus), gamma(gamma) {}
  Real density, viscosity, bulk_modulus, gamma;
  pmpm_material desc() const {
    pmpm_material m;
    check(pmpm_material_newton_fluid(density, viscosity, bulk_modulus, gamma, &m), "NewtonFluid");
    return m;
  }
};
struct DruckerPrager {
  DruckerPrager(Real density, Real E, Real pois, Real friction_angle, Real dilatancy_angle, Real cohesion)
      : density(density), E(E), pois(pois), friction_angle(friction_angle), dilatancy_angle(dilatancy_angle),
        cohesion(cohesion) {}
  Real density, E, pois, friction_angle, dilatancy_angle, cohesion;
  pmpm_material desc() const {
    pmpm_material m;
    check(pmpm_material_drucker_prager(density, E, pois, friction_angle, dilatancy_angle, cohesion, &m),
          "DruckerPrager");
    return m;
  }
  // DP_rheo::calculate_timestep (src/materials/dp_rheo.cpp:165-175): the
  // moduli are arguments there; these default to the material's own
  Real calculate_timestep(Real cell_size, Real factor) const {
    pmpm_material m = desc();
    Real dt;
    check(pmpm_material_timestep(&m, cell_size, factor, &dt), "calculate_timestep");
    return dt;
  }
};
// VonMises (src/materials/vonmises.cpp:31-44), 3D only
struct VonMises {
  VonMises(Real density, Real E, Real pois, Real yield_stress, Real H)
      : density(density), E(E), pois(pois), yield_stress(yield_stress), H(H) {
    bulk_modulus = E / (3.0f * (1.0f - 2.0f * pois));
    shear_modulus = E / (2.0f * (1.0f + pois));
  }
  Real density, E, pois, yield_stress, H, bulk_modulus, shear_modulus;
  pmpm_material desc() const {
    pmpm_material m;
    check(pmpm_material_von_mises(density, E, pois, yield_stress, H, &m), "VonMises");
    return m;
  }
  // VonMises::calculate_timestep (src/materials/vonmises.cpp:96-104)
  Real calculate_timestep(Real cell_size, Real factor) const {
    Real dt;
    check(pmpm_calculate_timestep(cell_size, factor, bulk_modulus, shear_modulus, density, &dt), "calculate_timestep");
    return dt;
  }
};
// ModifiedCamClay (src/materials/modifiedcamclay.cpp:47-63): the
// constructor's R is the preconsolidation ratio (pc = R p0 at the solver's
// initialize, from the particles' stresses); beta is kept and unused, as in
// the reference's stress update.
struct ModifiedCamClay {
  ModifiedCamClay(Real density, Real E, Real pois, Real M, Real lam, Real kap, Real Vs, Real R, Real Pt, Real beta)
      : density(density), E(E), pois(pois), M(M), lam(lam), kap(kap), Vs(Vs), R(R), Pt(Pt), beta(beta) {
    bulk_modulus = E / (3.0f * (1.0f - 2.0f * pois));
    shear_modulus = E / (2.0f * (1.0f + pois));
    lame_modulus = E * pois / ((1.0f + pois) * (1.0f - 2.0f * pois));
  }
  Real density, E, pois, M, lam, kap, Vs, R, Pt, beta, bulk_modulus, shear_modulus, lame_modulus;
  pmpm_material desc() const {
    pmpm_material m;
    check(pmpm_material_modified_cam_clay(density, E, pois, M, lam, kap, Vs, R, Pt, beta, &m), "ModifiedCamClay");
    return m;
  }
  // ModifiedCamClay::calculate_timestep (src/materials/modifiedcamclay.cpp:
  // 184-195): the moduli and density are arguments
  static Real calculate_timestep(Real cell_size, Real factor, Real bulk_modulus, Real shear_modulus, Real density) {
    Real dt;
    check(pmpm_calculate_timestep(cell_size, factor, bulk_modulus, shear_modulus, density, &dt), "calculate_timestep");
    return dt;
  }
};
// DruckerPragerCap (src/materials/druckerprager_cap.cpp:43-67): the
// ModifiedCamClay parameters plus the dilatancy angle in degrees
struct DruckerPragerCap : ModifiedCamClay {
  DruckerPragerCap(Real density, Real E, Real pois, Real M, Real lam, Real kap, Real Vs, Real R, Real Pt, Real beta,
                   Real dilatancy_angle)
      : ModifiedCamClay(density, E, pois, M, lam, kap, Vs, R, Pt, beta), dilatancy_angle(dilatancy_angle) {}
  Real dilatancy_angle;
  pmpm_material desc() const {
    pmpm_material m;
    check(pmpm_material_drucker_prager_cap(density, E, pois, M, lam, kap, Vs, R, Pt, beta, dilatancy_angle, &m),
          "DruckerPragerCap");
    return m;
  }
};
using MaterialType =
    std::variant<Material, LinearElastic, NewtonFluid, DruckerPrager, VonMises, ModifiedCamClay, DruckerPragerCap>;

struct BoundaryCondition {
  bool isActive = true;
  pmpm_bc desc(int) const {
    pmpm_bc b{};
    b.type = PMPM_BC_NODEDOMAIN;  // a NodeDomain with no constrained faces is inert
    for (int k = 0; k < 6; k++) b.ints[k] = -1;
    return b;
  }
};
struct Gravity {
  Gravity(const Vectorr &gravity, bool is_ramp, int ramp_step, const Vectorr &gravity_end)
      : gravity(gravity), is_ramp(is_ramp), ramp_step(ramp_step), gravity_end(gravity_end) {}
  Vectorr gravity;
  bool is_ramp;
  int ramp_step;
  Vectorr gravity_end;
  pmpm_bc desc(int) const {
    pmpm_bc b;
    check(pmpm_bc_gravity(gravity.data(), is_ramp ? 1 : 0, ramp_step, gravity_end.data(), DIM, &b), "Gravity");
    return b;
  }
};
struct NodeDomain {
  NodeDomain(const Vectori &face0_mode, const Vectori &face1_mode) : face0_mode(face0_mode), face1_mode(face1_mode) {}
  Vectori face0_mode, face1_mode;
  pmpm_bc desc(int) const {
    pmpm_bc b;
    check(pmpm_bc_nodedomain(face0_mode.data(), face1_mode.data(), DIM, &b), "NodeDomain");
    return b;
  }
};
struct BodyForce {
  BodyForce(const std::string &mode, const std::vector<Real> &values, const std::vector<bool> &mask)
      : values(values) {
    // BodyForce::BodyForce (src/boundaryconditions/bodyforce.cpp:44-61)
    mode_id = mode == "forces" ? 0 : (mode == "moments" ? 1 : (mode == "fixed" ? 2 : -1));
    if (mode_id < 0) throw std::invalid_argument("mode must be \"forces\", \"moments\" or \"fixed\"");
    for (bool m : mask) this->mask.push_back(m ? 1 : 0);
  }
  int mode_id;
  bool isActive = true;
  std::vector<Real> values;
  std::vector<unsigned char> mask;
  pmpm_bc desc(int num_nodes) const {
    if (values.size() != (size_t)num_nodes * DIM || mask.size() != (size_t)num_nodes)
      throw std::invalid_argument("BodyForce values/mask do not match the node count");
    pmpm_bc b;
    check(pmpm_bc_bodyforce(mode_id, values.data(), mask.data(), &b), "BodyForce");
    b.ints[1] = isActive ? 1 : 0;
    return b;
  }
};
struct PlanarDomain {
  PlanarDomain(const Vectorr &face0_friction, const Vectorr &face1_friction)
      : face0_friction(face0_friction), face1_friction(face1_friction) {}
  Vectorr face0_friction, face1_friction;  // degrees
  pmpm_bc desc(int) const {
    pmpm_bc b;
    check(pmpm_bc_planardomain(face0_friction.data(), face1_friction.data(), DIM, &b), "PlanarDomain");
    return b;
  }
};
// RigidBodyLevelSet (include/pyroclastmpm/boundaryconditions/rigidbodylevelset.h:
// 85-170): the reference's nearest-rigid-particle contact (STATIC, or
// set_mode_loop_rotate), or, once a shape is set, an analytic body with
// Coulomb friction (set_shape_sphere / set_shape_half_cylinder_shell,
// set_motion, set_friction).
struct RigidBodyLevelSet {
  RigidBodyLevelSet() { COM.fill(0.0f), euler_angles_per_second.fill(0.0f), center.fill(0.0f), velocity.fill(0.0f); }
  void set_mode_loop_rotate(const Vectorr &rate, const Vectorr &com) {
    mode = PMPM_RIGID_LOOP_ROTATE;
    euler_angles_per_second = rate;
    COM = com;
  }
  void set_shape_sphere(const Vectorr &c, Real radius) {
    shape = PMPM_SDF_SPHERE;
    center = c;
    dims = {radius, 0.0f, 0.0f};
  }
  void set_shape_half_cylinder_shell(const Vectorr &c, int ax, Real radius, Real thickness, Real length,
                                     Real angle0) {
    shape = PMPM_SDF_HALF_CYLINDER_SHELL;
    center = c;
    axis = ax;
    dims = {radius, thickness, length};
    angle = angle0;
  }
  void set_motion(const Vectorr &v, Real w) {
    velocity = v;
    angular_velocity = w;
  }
  int mode = PMPM_RIGID_STATIC;
  bool corrected_rotation = false;
  Vectorr euler_angles_per_second, COM;
  int shape = -1, axis = 1;
  Vectorr center, velocity;
  std::array<Real, 3> dims{0.0f, 0.0f, 0.0f};
  Real angle = 0.0f, angular_velocity = 0.0f, friction = 0.0f, contact_distance = 0.0f;
  pmpm_bc desc(int) const {
    pmpm_bc b;
    if (shape < 0)
      check(pmpm_bc_rigidbodylevelset(mode, euler_angles_per_second.data(), COM.data(), corrected_rotation ? 1 : 0,
                                      DIM, &b),
            "RigidBodyLevelSet");
    else
      check(pmpm_bc_rigid_sdf(shape, axis, center.data(), velocity.data(), angular_velocity, angle, dims.data(),
                              friction, contact_distance, DIM, &b),
            "RigidBodyLevelSet");
    return b;
  }
};
using BoundaryConditionType =
    std::variant<BoundaryCondition, Gravity, NodeDomain, BodyForce, PlanarDomain, RigidBodyLevelSet>;

// ---------------------------------------------------------------------------
// solvers
// ---------------------------------------------------------------------------
class Solver {
 public:
  Solver(const ParticlesContainer &p, const NodesContainer &n, const std::vector<MaterialType> &mats,
         const std::vector<BoundaryConditionType> &bcs, Real alpha = 0.99f, unsigned flags = 0)
      : nodes(n), particles(p), materials(mats), boundaryconditions(bcs) {
    // Solver::Solver (src/solver/solver.cpp:69-104): copies, partition,
    // initial volumes and masses
    pmpm_desc d{};
    d.dim = DIM;
    for (int a = 0; a < DIM; a++) {
      d.origin[a] = nodes.origin[a];
      d.end[a] = nodes.end[a];
    }
    d.cell_size = nodes.cell_size;
    d.shape_function = globals().shape_function;
    d.dt = globals().dt;
    d.particles_per_cell = globals().particles_per_cell;
    d.alpha = alpha;
    d.flags = flags | PMPM_FLAG_KEEP_VELOCITY_GRADIENT;
    d.resort_interval = 32;
    std::vector<pmpm_material> md;
    for (auto &m : materials) md.push_back(std::visit([](auto &x) { return x.desc(); }, m));
    std::vector<pmpm_bc> bd;
    for (auto &b : boundaryconditions) bd.push_back(std::visit([&](auto &x) { return x.desc(nodes.num_cells_total); }, b));
    d.num_materials = (int)md.size();
    d.materials = md.data();
    d.num_bcs = (int)bd.size();
    d.bcs = bd.data();
    handle = std::make_shared<SimHandle>();
    check(pmpm_create(&d, &handle->sim), "pmpm_create");
    const int D = DIM;
    const int nrig = (int)(particles.rigid_positions_.size() / D);
    const int nnon = (int)(particles.positions_.size() / D);
    check(pmpm_set_particles(handle->sim, nnon, particles.positions_.empty() ? nullptr : particles.positions_.data(),
                             particles.velocities_.empty() ? nullptr : particles.velocities_.data(),
                             particles.colors_.empty() ? nullptr : particles.colors_.data(), nrig,
                             particles.rigid_positions_.empty() ? nullptr : particles.rigid_positions_.data(),
                             particles.rigid_velocities_.empty() ? nullptr : particles.rigid_velocities_.data(),
                             particles.rigid_colors_.empty() ? nullptr : particles.rigid_colors_.data()),
          "pmpm_set_particles");
    particles.handle = handle;
    nodes.handle = handle;
    particles.apply_pending();
    check(pmpm_set_step(handle->sim, globals().step), "pmpm_set_step");
    check(pmpm_initialize(handle->sim), "pmpm_initialize");
    output();
  }
  virtual ~Solver() = default;

  // USL::solve + increment_global
  virtual void solve() {
    check(pmpm_solve(handle->sim, 1), "solve");
    sync_step();
  }
  // Solver::solve_nsteps (src/solver/solver.cpp:125-134)
  void solve_nsteps(int n) {
    check(pmpm_solve(handle->sim, n), "solve_nsteps");
    sync_step();
    output();
  }
  // Solver::run (src/solver/solver.cpp:140-174): output, solve, then
  // total_steps solves with output every output_frequency
  void run(int total_steps, int output_frequency) {
    output();
    const bool any = !particles.output_formats.empty() || !nodes.output_formats.empty();
    if (!any || output_frequency <= 0) {
      check(pmpm_solve(handle->sim, total_steps + 1), "run");
      sync_step();
      return;
    }
    check(pmpm_solve(handle->sim, 1), "run");
    for (int step = 1; step < total_steps + 1; step++) {
      // the reference writes after solve() and before the step increment
      check(pmpm_solve(handle->sim, 1), "run");
      if (step % output_frequency == 0) {
        int st = 0;
        check(pmpm_get_step(handle->sim, &st), "step");
        write_output(st - 1);
      }
    }
    sync_step();
  }
  // Solver::output (src/solver/solver.cpp:177-197)
  void output() { write_output(current_step()); }
  void stress_update() { check(pmpm_stress_update(handle->sim), "stress_update"); }
  int status() { return pmpm_synchronize(handle->sim); }
  int current_step() const {
    int s = 0;
    check(pmpm_get_step(handle->sim, &s), "step");
    return s;
  }

  NodesContainer nodes;
  ParticlesContainer particles;
  std::vector<MaterialType> materials;

  void write_output(int step) {
    const double time = (double)((Real)step * globals().dt);
    particles.output_vtk(step, time, globals().output_directory);
    nodes.output_vtk(step, time, globals().output_directory);
  }
  std::vector<BoundaryConditionType> boundaryconditions;
  std::shared_ptr<SimHandle> handle;

 protected:
  void sync_step() {
    globals().step = current_step();
    const int st = pmpm_synchronize(handle->sim);
    if (st != PMPM_OK && st != PMPM_ERR_OUT_OF_DOMAIN) check(st, "step");
  }
};

class USL : public Solver {
 public:
  USL(const ParticlesContainer &p, const NodesContainer &n, const std::vector<MaterialType> &mats,
      const std::vector<BoundaryConditionType> &bcs, Real alpha = 0.99f, unsigned flags = 0)
      : Solver(p, n, mats, bcs, alpha, flags), alpha(alpha) {}
  // USL::P2G / USL::G2P (src/solver/usl/usl.cpp:118-199), after a partition
  void partition() { check(pmpm_partition(handle->sim), "partition"); }
  void P2G() { check(pmpm_p2g(handle->sim, 0), "P2G"); }
  void G2P() { check(pmpm_g2p(handle->sim, 0), "G2P"); }
  Real alpha;
};

// MUSL (include/pyroclastmpm/solver/musl/musl.cuh: declared by the reference,
// not built there): USL's P2G and grid update, then G2P_double_mapping,
// P2G_double_mapping and G2P (velocity gradient from the remapped momenta).
class MUSL : public USL {
 public:
  MUSL(const ParticlesContainer &p, const NodesContainer &n, const std::vector<MaterialType> &mats,
       const std::vector<BoundaryConditionType> &bcs, Real alpha = 0.99f, unsigned flags = 0)
      : USL(p, n, mats, bcs, alpha, flags | PMPM_FLAG_MUSL) {}
  void G2P_double_mapping() { check(pmpm_musl_stage(handle->sim, 1), "G2P_double_mapping"); }
  void P2G_double_mapping() { check(pmpm_musl_stage(handle->sim, 2), "P2G_double_mapping"); }
  void G2P() { check(pmpm_musl_stage(handle->sim, 3), "G2P"); }
};

}  // namespace dim2 / dim3
}  // namespace pyroclastmpm
