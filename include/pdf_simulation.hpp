/*
 * pdf_simulation.hpp — C++ front of the B200 step loop with the reference's
 * simulation-building interface, over the C ABI of pdf.h (header only).
 *
 * The reference's caller (src/main.cpp:40-124) reads a scene and the
 * simulation parameters from JSON, builds the simulation with getSimulation
 * and drives it with step() and exportStats():
 *
 *   PhysicScene scene = getSceneFromJSONFileName(path);             // scene_building.hpp:37
 *   SimulationParameters params =
 *       getSimulationParametersFromJSONFileName(path);              // simulation_building.hpp:53
 *   std::unique_ptr<SimulationBase> sim = getSimulation(scene, params);  // simulation_building.hpp:70
 *   for (...) sim->step();                                          // SimulationBase.hpp:70
 *   sim->exportStats(of);                                           // SimulationBase.hpp:117
 *
 * The same calls here (namespace pdf) build and drive the device step loop:
 * PhysicScene owns the loaded scene, SimulationParameters the parameters,
 * getSimulation returns a std::unique_ptr<SimulationGpu> whose step() and
 * exportStats(std::ofstream&) replace SimulationBase's (the reference always
 * builds SimulationFrictionEstimation: simulation_building.cpp:94-97).  Where
 * the reference's caller reads the state back through the scene's meshes
 * (PhysicMesh::getGeneralizedPositions / Speeds), the simulation hands it out
 * here, since the device holds it.  Errors surface as pdf::Error (a
 * std::runtime_error carrying the pdf_status) instead of the reference's
 * std::invalid_argument for configuration errors and silent solver failures.
 */
#ifndef PDF_SIMULATION_HPP
#define PDF_SIMULATION_HPP

#include <cstdint>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "pdf.h"

namespace pdf {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int status() const noexcept { return status_; }

 private:
  int status_;
};

inline void check(int status, const pdf_handle* h = nullptr) {
  if (status != PDF_OK) throw Error(status, h ? pdf_last_error(h) : pdf_global_error());
}

/* A scene read from the reference's JSON format (getSceneFromJSONDocument,
 * src/scene_building.cpp:279-318). */
class PhysicScene {
 public:
  explicit PhysicScene(const std::string& json_path) {
    pdf_scene* s = nullptr;
    check(pdf_scene_load_json(json_path.c_str(), &s));
    scene_.reset(s);
  }
  pdf_scene_desc desc() const {
    pdf_scene_desc d{};
    check(pdf_scene_view(scene_.get(), &d));
    return d;
  }
  int32_t getNumberOfVertices() const { return desc().n_vertices; }

 private:
  struct Free {
    void operator()(pdf_scene* s) const { pdf_scene_free(s); }
  };
  std::unique_ptr<pdf_scene, Free> scene_;
};

/* getSimulationParametersFromJSONDocument (src/simulation_building.cpp:37-78):
 * the step-loop parameters plus the driver's frame count and steps per frame. */
struct SimulationParameters {
  pdf_params params{};
  int32_t max_output_frame = 0;
  int32_t sim_steps_per_frame = 1;
};

inline PhysicScene getSceneFromJSONFileName(const char* filename) { return PhysicScene(filename); }

inline SimulationParameters getSimulationParametersFromJSONFileName(const char* filename) {
  SimulationParameters p;
  check(pdf_params_load_json(filename, &p.params, &p.max_output_frame, &p.sim_steps_per_frame));
  return p;
}

/* The device step loop behind the reference's SimulationBase interface. */
class SimulationGpu {
 public:
  SimulationGpu(const PhysicScene& scene, const SimulationParameters& params) {
    const pdf_scene_desc d = scene.desc();
    n_ = d.n_vertices;
    pdf_handle* h = nullptr;
    check(pdf_create(&d, &params.params, &h));
    h_.reset(h);
  }

  /* SimulationBase::step() (SimulationBase.cpp:103-173). */
  void step() { check(pdf_step(h_.get(), 1, nullptr), h_.get()); }

  /* SimulationBase::exportStats(std::ofstream&) (SFE:756-771): appends the
   * stats sections to the stream. */
  void exportStats(std::ofstream& of) const {
    int64_t len = 0;
    check(pdf_export_stats_text(h_.get(), nullptr, 0, &len), h_.get());
    std::string text((size_t)len + 1, '\0');
    check(pdf_export_stats_text(h_.get(), &text[0], len + 1, &len), h_.get());
    text.resize((size_t)len);
    of << text;
  }

  /* The scene's generalized positions / speeds (3N, vertex-major), as the
   * reference's caller reads them from the PhysicMesh after a step. */
  std::vector<double> getGeneralizedPositions() const {
    std::vector<double> q(3 * (size_t)n_);
    check(pdf_get_state(h_.get(), q.data(), nullptr), h_.get());
    return q;
  }
  std::vector<double> getGeneralizedSpeeds() const {
    std::vector<double> v(3 * (size_t)n_);
    check(pdf_get_state(h_.get(), nullptr, v.data()), h_.get());
    return v;
  }
  void setGeneralizedPositions(const std::vector<double>& q) {
    check(pdf_set_state(h_.get(), q.data(), nullptr), h_.get());
  }
  void setGeneralizedSpeeds(const std::vector<double>& v) {
    check(pdf_set_state(h_.get(), nullptr, v.data()), h_.get());
  }
  pdf_handle* handle() const { return h_.get(); }

 private:
  struct Destroy {
    void operator()(pdf_handle* h) const { pdf_destroy(h); }
  };
  std::unique_ptr<pdf_handle, Destroy> h_;
  int32_t n_ = 0;
};

/* getSimulation (src/simulation_building.cpp:80-98). */
inline std::unique_ptr<SimulationGpu> getSimulation(const PhysicScene& scene, const SimulationParameters& params) {
  return std::unique_ptr<SimulationGpu>(new SimulationGpu(scene, params));
}

}  // namespace pdf

#endif /* PDF_SIMULATION_HPP */
