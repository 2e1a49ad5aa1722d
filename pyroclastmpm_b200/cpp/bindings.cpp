// pybind11 module with the reference's Python API (python/pybind/**): module
// MPM2D or MPM3D (-DDIM), classes and argument names as the reference binds
// them.  Arrays cross as numpy arrays (the reference returns lists of Eigen
// vectors; np.asarray of either gives the same [n, dim] array).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "pyroclastmpm.hpp"

namespace py = pybind11;
using namespace pyroclastmpm;

#if DIM == 2
#define PMPM_MODULE MPM2D
#else
#define PMPM_MODULE MPM3D
#endif

namespace {

using farr = py::array_t<float, py::array::c_style | py::array::forcecast>;
using iarr = py::array_t<int, py::array::c_style | py::array::forcecast>;

std::vector<float> flat(const py::object &o, size_t per) {
  if (o.is_none()) return {};
  farr a = farr::ensure(o);
  if (!a) throw std::invalid_argument("expected an array of numbers");
  if (a.size() == 0) return {};
  if ((size_t)a.size() % per) throw std::invalid_argument("array size is not a multiple of the dimension");
  return std::vector<float>(a.data(), a.data() + a.size());
}
std::vector<int> flati(const py::object &o) {
  if (o.is_none()) return {};
  iarr a = iarr::ensure(o);
  if (!a || a.size() == 0) return {};
  return std::vector<int>(a.data(), a.data() + a.size());
}
template <typename V>
V vec(const py::object &o) {
  V v{};
  auto f = flat(o, 1);
  for (size_t k = 0; k < v.size() && k < f.size(); k++) v[k] = (typename V::value_type)f[k];
  return v;
}
template <typename T>
py::array_t<T> to_array(const std::vector<T> &v, std::vector<py::ssize_t> shape) {
  py::array_t<T> out(shape);
  std::copy(v.begin(), v.end(), out.mutable_data());
  return out;
}

}  // namespace

PYBIND11_MODULE(PMPM_MODULE, m) {
  m.doc() = "B200-native USL MPM step with the PyroclastMPM Python API";
  m.attr("global_dimension") = DIM;

  m.def("set_globals", &set_globals, py::arg("time_step"), py::arg("particles_per_cell"),
        py::arg("shape_function") = "linear", py::arg("output_directory") = "./output/");
  m.def("set_global_shapefunction", &set_global_shapefunction, py::arg("shapefunction") = "linear");
  m.def("set_global_timestep", &set_global_timestep, py::arg("timestep"));
  m.def("set_global_step", &set_global_step, py::arg("step"));
  m.def("set_global_output_directory", &set_global_output_directory, py::arg("directory"));

  py::class_<NodesContainer>(m, "NodesContainer")
      .def(py::init([](py::object o, py::object e, float h) {
             return NodesContainer(vec<Vectorr>(o), vec<Vectorr>(e), h);
           }),
           py::arg("origin"), py::arg("end"), py::arg("cell_size"))
      .def("give_coords", [](const NodesContainer &n) {
        return to_array(n.give_coords(), {n.num_cells_total, DIM});
      })
      .def_property_readonly("num_cells", [](const NodesContainer &n) { return n.num_cells; })
      .def_property_readonly("num_cells_total", [](const NodesContainer &n) { return n.num_cells_total; })
      .def_property_readonly("masses", [](const NodesContainer &n) { return to_array(n.masses(), {n.num_cells_total}); })
      .def_property_readonly("moments",
                             [](const NodesContainer &n) { return to_array(n.moments(), {n.num_cells_total, DIM}); })
      .def_property_readonly("moments_nt", [](const NodesContainer &n) {
        return to_array(n.moments_nt(), {n.num_cells_total, DIM});
      })
      .def(
          "set_output_formats",
          [](NodesContainer &n, const std::vector<std::string> &f) { n.output_formats = f; },
          py::arg("output_formats"))
      .def_readwrite("output_formats", &NodesContainer::output_formats);

  auto P = py::class_<ParticlesContainer>(m, "ParticlesContainer", py::dynamic_attr());
  P.def(py::init([](py::object pos, py::object vel, py::object col, py::object rpos, py::object rvel, py::object rcol) {
          return ParticlesContainer(flat(pos, DIM), flat(vel, DIM), flati(col), flat(rpos, DIM), flat(rvel, DIM),
                                    flati(rcol));
        }),
        py::arg("positions"), py::arg("velocities") = py::none(), py::arg("colors") = py::none(),
        py::arg("rigid_positions") = py::none(), py::arg("rigid_velocities") = py::none(),
        py::arg("rigid_colors") = py::none());
  P.def_readonly("num_particles", &ParticlesContainer::num_particles);
  P.def(
      "set_output_formats", [](ParticlesContainer &p, const std::vector<std::string> &f) { p.output_formats = f; },
      py::arg("output_formats"));
  P.def_readwrite("output_formats", &ParticlesContainer::output_formats);
  P.def_readwrite("exclude_rigid_from_output", &ParticlesContainer::exclude_rigid_from_output);
  // pickle_save_particles / pickle_load_particles (python/pybind/particles/
  // particles_bind.cpp:39-83): the same 13-entry tuple; psi and dpsi are not
  // kept between steps here (they are recomputed in registers), so entries
  // 10 and 12 are empty
  P.def(py::pickle(
      [](ParticlesContainer &p) {
        const bool bound = (bool)p.handle;
        auto getf = [&](int id, int nc, const std::vector<Real> &host) -> py::array_t<float> {
          if (bound) return to_array(p.get<float>(id, nc), {p.num_particles, nc});
          if (!host.empty()) return to_array(host, {(py::ssize_t)(host.size() / nc), nc});
          return py::array_t<float>(std::vector<py::ssize_t>{0, nc});
        };
        std::vector<Real> pos = p.positions_, vel = p.velocities_;
        pos.insert(pos.end(), p.rigid_positions_.begin(), p.rigid_positions_.end());
        py::array_t<float> x = getf(PMPM_FIELD_POSITIONS, DIM, pos);
        py::array_t<float> v = bound ? getf(PMPM_FIELD_VELOCITIES, DIM, {}) : py::array_t<float>();
        if (!bound) {
          std::vector<Real> vv = p.velocities_;
          const size_t nn = p.positions_.size() / DIM, nr = p.rigid_positions_.size() / DIM;
          if (vv.empty()) vv.assign(nn * DIM, 0.0f);
          if (p.rigid_velocities_.empty())
            vv.insert(vv.end(), nr * DIM, 0.0f);
          else
            vv.insert(vv.end(), p.rigid_velocities_.begin(), p.rigid_velocities_.end());
          v = to_array(vv, {(py::ssize_t)(nn + nr), DIM});
        }
        std::vector<int> col, rig;
        if (bound) {
          for (auto c : p.get<unsigned char>(PMPM_FIELD_COLORS, 1)) col.push_back(c);
          for (auto r : p.get<unsigned char>(PMPM_FIELD_IS_RIGID, 1)) rig.push_back(r);
        } else {
          const size_t nn = p.positions_.size() / DIM, nr = p.rigid_positions_.size() / DIM;
          for (size_t i = 0; i < nn; i++) col.push_back(i < p.colors_.size() ? p.colors_[i] : 0);
          for (size_t i = 0; i < nr; i++) col.push_back(i < p.rigid_colors_.size() ? p.rigid_colors_[i] : 0);
          rig.assign(nn, 0);
          rig.insert(rig.end(), nr, 1);
        }
        auto opt = [&](int id, int nc) -> py::object {
          if (!bound) return py::list();
          return getf(id, nc, {});
        };
        return py::make_tuple(x, v, col, rig, opt(PMPM_FIELD_STRESSES, 9), opt(PMPM_FIELD_MASSES, 1),
                              opt(PMPM_FIELD_VOLUMES, 1), p.output_formats, opt(PMPM_FIELD_F, DIM * DIM),
                              opt(PMPM_FIELD_VELOCITY_GRADIENT, DIM * DIM), py::list(),
                              opt(PMPM_FIELD_VOLUMES_ORIGINAL, 1), py::list());
      },
      [](py::tuple t) {
        if (t.size() != 13) throw std::runtime_error("a ParticlesContainer pickle is a 13-entry tuple");
        auto x = flat(t[0], DIM), v = flat(t[1], DIM);
        auto col = t[2].cast<std::vector<int>>();
        auto rig = t[3].cast<std::vector<int>>();
        const size_t n = x.size() / DIM;
        std::vector<Real> xp, vp, xr, vr;
        std::vector<int> cp, cr;
        for (size_t i = 0; i < n; i++) {
          const bool r = i < rig.size() && rig[i];
          auto &X = r ? xr : xp;
          auto &Vv = r ? vr : vp;
          for (int a = 0; a < DIM; a++) {
            X.push_back(x[i * DIM + a]);
            Vv.push_back(v.empty() ? 0.0f : v[i * DIM + a]);
          }
          (r ? cr : cp).push_back(i < col.size() ? col[i] : 0);
        }
        ParticlesContainer p(xp, vp, cp, xr, vr, cr);
        // stored fields are in input order: non-rigid first, then rigid
        std::vector<size_t> order;
        for (size_t i = 0; i < n; i++)
          if (!(i < rig.size() && rig[i])) order.push_back(i);
        for (size_t i = 0; i < n; i++)
          if (i < rig.size() && rig[i]) order.push_back(i);
        auto put = [&](int id, int nc, py::handle h) {
          auto f = flat(py::reinterpret_borrow<py::object>(h), 1);
          if (f.size() != n * nc) return;  // not stored
          std::vector<float> o(n * nc);
          for (size_t j = 0; j < n; j++)
            for (int k = 0; k < nc; k++) o[j * nc + k] = f[order[j] * nc + k];
          p.set<float>(id, o, nc);
        };
        put(PMPM_FIELD_STRESSES, 9, t[4]);
        put(PMPM_FIELD_MASSES, 1, t[5]);
        put(PMPM_FIELD_VOLUMES, 1, t[6]);
        p.output_formats = t[7].cast<std::vector<std::string>>();
        put(PMPM_FIELD_F, DIM * DIM, t[8]);
        put(PMPM_FIELD_VELOCITY_GRADIENT, DIM * DIM, t[9]);
        put(PMPM_FIELD_VOLUMES_ORIGINAL, 1, t[11]);
        return p;
      }));
#define PMPM_PROP(NAME, ID, NCOMP, ...)                                                              \
  P.def_property(                                                                                   \
      NAME,                                                                                         \
      [](ParticlesContainer &p) { return to_array(p.get<float>(ID, NCOMP), {__VA_ARGS__}); },       \
      [](ParticlesContainer &p, py::object v) { p.set<float>(ID, flat(v, 1), NCOMP); })
  PMPM_PROP("positions", PMPM_FIELD_POSITIONS, DIM, p.num_particles, DIM);
  PMPM_PROP("velocities", PMPM_FIELD_VELOCITIES, DIM, p.num_particles, DIM);
  PMPM_PROP("stresses", PMPM_FIELD_STRESSES, 9, p.num_particles, 3, 3);
  PMPM_PROP("F", PMPM_FIELD_F, DIM * DIM, p.num_particles, DIM, DIM);
  PMPM_PROP("velocity_gradient", PMPM_FIELD_VELOCITY_GRADIENT, DIM * DIM, p.num_particles, DIM, DIM);
  PMPM_PROP("masses", PMPM_FIELD_MASSES, 1, p.num_particles);
  PMPM_PROP("volumes", PMPM_FIELD_VOLUMES, 1, p.num_particles);
  PMPM_PROP("volumes_original", PMPM_FIELD_VOLUMES_ORIGINAL, 1, p.num_particles);
#undef PMPM_PROP
  P.def_property(
      "colors",
      [](ParticlesContainer &p) {
        auto c = p.get<unsigned char>(PMPM_FIELD_COLORS, 1);
        return to_array(std::vector<int>(c.begin(), c.end()), {p.num_particles});
      },
      [](ParticlesContainer &p, py::object v) {
        auto c = flati(v);
        p.set<unsigned char>(PMPM_FIELD_COLORS, std::vector<unsigned char>(c.begin(), c.end()), 1);
      });

  py::class_<Material>(m, "Material", py::dynamic_attr()).def(py::init<>()).def_readwrite("density", &Material::density);
  py::class_<LinearElastic>(m, "LinearElastic", py::dynamic_attr())
      .def(py::init<float, float, float>(), py::arg("density"), py::arg("E"), py::arg("pois") = 0.0f)
      .def_readonly("E", &LinearElastic::E)
      .def_readonly("pois", &LinearElastic::pois)
      .def_readonly("shear_modulus", &LinearElastic::shear_modulus)
      .def_readonly("lame_modulus", &LinearElastic::lame_modulus)
      .def_readonly("bulk_modulus", &LinearElastic::bulk_modulus)
      .def_readwrite("density", &LinearElastic::density)
      .def_readwrite("corrected", &LinearElastic::corrected)
      .def("calculate_timestep", &LinearElastic::calculate_timestep, py::arg("cell_size"), py::arg("factor"));
  py::class_<NewtonFluid>(m, "NewtonFluid", py::dynamic_attr())
      .def(py::init<float, float, float, float>(), py::arg("density"), py::arg("viscosity"),
           py::arg("bulk_modulus") = 0.0f, py::arg("gamma") = 7.0f)
      .def_readwrite("density", &NewtonFluid::density)
      .def_readwrite("viscosity", &NewtonFluid::viscosity)
      .def_readwrite("bulk_modulus", &NewtonFluid::bulk_modulus)
      .def_readwrite("gamma", &NewtonFluid::gamma);
  py::class_<DruckerPrager>(m, "DruckerPrager", py::dynamic_attr())
      .def(py::init<float, float, float, float, float, float>(), py::arg("density"), py::arg("E"),
           py::arg("pois") = 0.0f, py::arg("friction_angle") = 30.0f, py::arg("dilatancy_angle") = 0.0f,
           py::arg("cohesion") = 0.0f)
      .def_readwrite("density", &DruckerPrager::density)
      .def("calculate_timestep", &DruckerPrager::calculate_timestep, py::arg("cell_size"), py::arg("factor"));

  py::class_<VonMises>(m, "VonMises", py::dynamic_attr())
      .def(py::init<float, float, float, float, float>(), py::arg("density"), py::arg("E"), py::arg("pois"),
           py::arg("yield_stress"), py::arg("H"))
      .def_readwrite("density", &VonMises::density)
      .def_readonly("E", &VonMises::E)
      .def_readonly("pois", &VonMises::pois)
      .def_readonly("yield_stress", &VonMises::yield_stress)
      .def_readonly("H", &VonMises::H)
      .def_readonly("bulk_modulus", &VonMises::bulk_modulus)
      .def_readonly("shear_modulus", &VonMises::shear_modulus)
      .def("calculate_timestep", &VonMises::calculate_timestep, py::arg("cell_size"), py::arg("factor"));

  py::class_<ModifiedCamClay>(m, "ModifiedCamClay", py::dynamic_attr())
      .def(py::init<float, float, float, float, float, float, float, float, float, float>(), py::arg("density"),
           py::arg("E"), py::arg("pois"), py::arg("M"), py::arg("lam"), py::arg("kap"), py::arg("Vs"), py::arg("R"),
           py::arg("Pt"), py::arg("beta"))
      // ModifiedCamClay::initialize (modified_camclay_bind.cpp): the history is
      // set up when the solver is built from the particles' current stresses
      .def("initialize",
           [](ModifiedCamClay &, ParticlesContainer particles, int mat_id) { return py::make_tuple(particles, mat_id); },
           py::arg("particles"), py::arg("mat_id") = 0)
      .def_readwrite("density", &ModifiedCamClay::density)
      .def_readonly("E", &ModifiedCamClay::E)
      .def_readonly("pois", &ModifiedCamClay::pois)
      .def_readonly("M", &ModifiedCamClay::M)
      .def_readonly("lam", &ModifiedCamClay::lam)
      .def_readonly("kap", &ModifiedCamClay::kap)
      .def_readonly("Vs", &ModifiedCamClay::Vs)
      .def_readonly("R", &ModifiedCamClay::R)
      .def_readonly("Pt", &ModifiedCamClay::Pt)
      .def_readonly("beta", &ModifiedCamClay::beta)
      .def_readonly("bulk_modulus", &ModifiedCamClay::bulk_modulus)
      .def_readonly("shear_modulus", &ModifiedCamClay::shear_modulus)
      .def_readonly("lame_modulus", &ModifiedCamClay::lame_modulus)
      .def_static("calculate_timestep", &ModifiedCamClay::calculate_timestep, py::arg("cell_size"), py::arg("factor"),
                  py::arg("bulk_modulus"), py::arg("shear_modulus"), py::arg("density"));

  py::class_<DruckerPragerCap>(m, "DruckerPragerCap", py::dynamic_attr())
      .def(py::init<float, float, float, float, float, float, float, float, float, float, float>(), py::arg("density"),
           py::arg("E"), py::arg("pois"), py::arg("M"), py::arg("lam"), py::arg("kap"), py::arg("Vs"), py::arg("R"),
           py::arg("Pt"), py::arg("beta"), py::arg("dilatancy_angle") = 0.0f)
      .def("initialize",
           [](DruckerPragerCap &, ParticlesContainer particles, int mat_id) { return py::make_tuple(particles, mat_id); },
           py::arg("particles"), py::arg("mat_id") = 0)
      .def_readwrite("density", &DruckerPragerCap::density)
      .def_readonly("E", &DruckerPragerCap::E)
      .def_readonly("pois", &DruckerPragerCap::pois)
      .def_readonly("M", &DruckerPragerCap::M)
      .def_readonly("lam", &DruckerPragerCap::lam)
      .def_readonly("kap", &DruckerPragerCap::kap)
      .def_readonly("Vs", &DruckerPragerCap::Vs)
      .def_readonly("R", &DruckerPragerCap::R)
      .def_readonly("Pt", &DruckerPragerCap::Pt)
      .def_readonly("beta", &DruckerPragerCap::beta)
      .def_readonly("dilatancy_angle", &DruckerPragerCap::dilatancy_angle)
      .def_readonly("bulk_modulus", &DruckerPragerCap::bulk_modulus)
      .def_readonly("shear_modulus", &DruckerPragerCap::shear_modulus);

  py::class_<BoundaryCondition>(m, "BoundaryCondition").def(py::init<>());
  py::class_<Gravity>(m, "Gravity", py::dynamic_attr())
      .def(py::init([](py::object g, bool is_ramp, int ramp_step, py::object ge) {
             return Gravity(vec<Vectorr>(g), is_ramp, ramp_step, vec<Vectorr>(ge));
           }),
           py::arg("gravity"), py::arg("is_ramp") = false, py::arg("ramp_step") = 0,
           py::arg("gravity_end") = py::none())
      .def_readwrite("gravity", &Gravity::gravity);
  py::class_<NodeDomain>(m, "NodeDomain", py::dynamic_attr())
      .def(py::init([](py::object f0, py::object f1) { return NodeDomain(vec<Vectori>(f0), vec<Vectori>(f1)); }),
           py::arg("face0_mode") = py::none(), py::arg("face1_mode") = py::none());
  py::class_<BodyForce>(m, "BodyForce", py::dynamic_attr())
      .def(py::init([](const std::string &mode, py::object values, py::object mask) {
             auto mk = flati(mask);
             return BodyForce(mode, flat(values, DIM), std::vector<bool>(mk.begin(), mk.end()));
           }),
           py::arg("mode"), py::arg("values"), py::arg("mask"))
      .def_readwrite("isActive", &BodyForce::isActive);
  py::class_<PlanarDomain>(m, "PlanarDomain", py::dynamic_attr())
      .def(py::init([](py::object f0, py::object f1) { return PlanarDomain(vec<Vectorr>(f0), vec<Vectorr>(f1)); }),
           py::arg("face0_friction") = py::none(), py::arg("face1_friction") = py::none());

  py::class_<RigidBodyLevelSet>(m, "RigidBodyLevelSet", py::dynamic_attr())
      .def(py::init<>())
      .def(
          "set_mode_loop_rotate",
          [](RigidBodyLevelSet &r, py::object rate, py::object com) {
            r.set_mode_loop_rotate(vec<Vectorr>(rate), vec<Vectorr>(com));
          },
          py::arg("euler_angles_per_second"), py::arg("COM") = py::none())
      .def(
          "set_shape_sphere", [](RigidBodyLevelSet &r, py::object c, float radius) { r.set_shape_sphere(vec<Vectorr>(c), radius); },
          py::arg("center"), py::arg("radius"))
      .def(
          "set_shape_half_cylinder_shell",
          [](RigidBodyLevelSet &r, py::object c, int axis, float radius, float thickness, float length, float angle) {
            r.set_shape_half_cylinder_shell(vec<Vectorr>(c), axis, radius, thickness, length, angle);
          },
          py::arg("center"), py::arg("axis"), py::arg("radius"), py::arg("thickness"), py::arg("length"),
          py::arg("angle") = 0.0f)
      .def(
          "set_motion", [](RigidBodyLevelSet &r, py::object v, float w) { r.set_motion(vec<Vectorr>(v), w); },
          py::arg("velocity"), py::arg("angular_velocity") = 0.0f)
      .def_readwrite("friction", &RigidBodyLevelSet::friction)
      .def_readwrite("contact_distance", &RigidBodyLevelSet::contact_distance)
      .def_readwrite("corrected_rotation", &RigidBodyLevelSet::corrected_rotation)
      .def("set_output_formats", [](RigidBodyLevelSet &, const std::vector<std::string> &) {},
           py::arg("output_formats"));

  m.def("calculate_timestep",
        [](float cell_size, float factor, float bulk, float shear, float density) {
          float dt;
          check(pmpm_calculate_timestep(cell_size, factor, bulk, shear, density, &dt), "calculate_timestep");
          return dt;
        },
        py::arg("cell_size"), py::arg("factor"), py::arg("bulk_modulus"), py::arg("shear_modulus"),
        py::arg("density"));

  py::class_<Solver>(m, "Solver")
      .def(py::init<ParticlesContainer, NodesContainer, std::vector<MaterialType>, std::vector<BoundaryConditionType>>(),
           py::arg("particles"), py::arg("nodes"), py::arg("materials") = std::vector<MaterialType>(),
           py::arg("boundaryconditions") = std::vector<BoundaryConditionType>())
      .def("run", &Solver::run, py::arg("total_steps"), py::arg("output_frequency"))
      .def("solve", &Solver::solve)
      .def("solve_nsteps", &Solver::solve_nsteps, py::arg("n_steps"))
      .def("stress_update", &Solver::stress_update)
      .def_property_readonly("current_step", &Solver::current_step)
      .def_readwrite("particles", &Solver::particles)
      .def_readwrite("nodes", &Solver::nodes);
  py::class_<USL, Solver>(m, "USL")
      .def(py::init<ParticlesContainer, NodesContainer, std::vector<MaterialType>, std::vector<BoundaryConditionType>,
                    float, unsigned>(),
           py::arg("particles"), py::arg("nodes"), py::arg("materials") = std::vector<MaterialType>(),
           py::arg("boundaryconditions") = std::vector<BoundaryConditionType>(), py::arg("alpha") = 0.99f,
           py::arg("flags") = 0u)
      .def("partition", &USL::partition)
      .def("P2G", &USL::P2G)
      .def("G2P", &USL::G2P)
      .def_readonly("alpha", &USL::alpha);
  py::class_<MUSL, USL>(m, "MUSL")
      .def(py::init<ParticlesContainer, NodesContainer, std::vector<MaterialType>, std::vector<BoundaryConditionType>,
                    float, unsigned>(),
           py::arg("particles"), py::arg("nodes"), py::arg("materials") = std::vector<MaterialType>(),
           py::arg("boundaryconditions") = std::vector<BoundaryConditionType>(), py::arg("alpha") = 0.99f,
           py::arg("flags") = 0u)
      .def("G2P_double_mapping", &MUSL::G2P_double_mapping)
      .def("P2G_double_mapping", &MUSL::P2G_double_mapping)
      .def("G2P", &MUSL::G2P);
}
