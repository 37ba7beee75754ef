// pdf_run — command-line driver of the step loop with the reference's
// observable behaviour (src/main.cpp:40-124), written against the C ABI of
// include/pdf.h only:
//   * output directory data<k> (the first that does not exist), the scene JSON
//     copied into it, frames in data<k>/output (initializeFileSystem,
//     src/physics/io.cpp:23-46; getOBJFilePath :61-69);
//   * "Time Step: i" before each step, the simulated time after it
//     (SimulationBase.cpp:160-161), the "log" callbacks
//     (src/log_building.cpp:89-118), one OBJ frame of mesh 0 every
//     "Steps per frame" steps starting with step 0 (Mesh::writeObj,
//     src/geometry/Mesh.cpp:95-109), progress milestones on stderr, stats.txt
//     at the end (exportStats);
//   * --print-alart-curnier prints every PD iteration's per-contact
//     Alart-Curnier norms like the reference built with
//     PRINT_ALART_CURNIER_ERROR (SFE:720-752).
// Frames are copied from the device asynchronously (pdf_frame_capture) and
// written by a second host thread while the GPU runs the following steps.
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <list>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pdf.h"

namespace fs = std::filesystem;

namespace {

[[noreturn]] void die(const std::string& what) {
  std::cerr << "pdf_run: " << what << std::endl;
  std::exit(EXIT_FAILURE);
}

void check(int status, pdf_handle* h, const char* what) {
  if (status != PDF_OK) die(std::string(what) + ": " + (h ? pdf_last_error(h) : pdf_global_error()));
}

// Eigen's default printing of a column vector: one coefficient per line,
// right-aligned to the widest coefficient as the stream formats it.
void print_column(std::ostream& os, const double* x) {
  std::string str[3];
  size_t width = 0;
  for (int k = 0; k < 3; ++k) {
    std::ostringstream ss;
    ss.copyfmt(os);
    ss << x[k];
    str[k] = ss.str();
    width = std::max(width, str[k].size());
  }
  for (int k = 0; k < 3; ++k) {
    if (k) os << "\n";
    os << std::string(width - str[k].size(), ' ') << str[k];
  }
}

// Mesh 0 as the reference's OBJ writer prints it: "v x y z" per vertex, then
// "f a b c" per triangle, 1-based, default stream formatting.
struct ObjWriter {
  int v0 = 0, nv = 0;
  std::vector<int32_t> tris;  // mesh-local
  void write(const fs::path& path, const double* q) const {
    std::ofstream of(path);
    if (!of) die("cannot write " + path.string());
    for (int i = 0; i < nv; ++i) {
      const double* x = q + 3 * (size_t)(v0 + i);
      of << "v " << x[0] << " " << x[1] << " " << x[2] << std::endl;
    }
    for (size_t t = 0; t < tris.size() / 3; ++t)
      of << "f " << tris[3 * t] + 1 << " " << tris[3 * t + 1] + 1 << " " << tris[3 * t + 2] + 1 << std::endl;
  }
};

// Frame writer thread: frames are handed over as (slot, frame number); the
// thread waits for the slot's device copy, writes the file and frees the slot.
class FrameWriter {
 public:
  FrameWriter(pdf_handle* h, const ObjWriter& obj, fs::path dir) : h_(h), obj_(obj), dir_(std::move(dir)) {
    th_ = std::thread([this] { run(); });
  }
  ~FrameWriter() { finish(); }
  // blocks until `slot` is free, then starts its copy and queues the frame
  void submit(int slot, size_t frame) {
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return !busy_[slot]; });
      busy_[slot] = true;
    }
    check(pdf_frame_capture(h_, slot), h_, "frame capture");
    {
      std::lock_guard<std::mutex> lk(mu_);
      queue_.emplace_back(slot, frame);
    }
    cv_.notify_all();
  }
  void finish() {
    if (!th_.joinable()) return;
    {
      std::lock_guard<std::mutex> lk(mu_);
      done_ = true;
    }
    cv_.notify_all();
    th_.join();
  }

 private:
  void run() {
    for (;;) {
      std::pair<int, size_t> job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return done_ || !queue_.empty(); });
        if (queue_.empty()) return;
        job = queue_.front();
        queue_.pop_front();
      }
      const double* q = nullptr;
      check(pdf_frame_wait(h_, job.first, &q), h_, "frame copy");
      std::ostringstream name;
      name << "out_" << std::setw(6) << std::setfill('0') << job.second << ".obj";
      obj_.write(dir_ / name.str(), q);
      {
        std::lock_guard<std::mutex> lk(mu_);
        busy_[job.first] = false;
      }
      cv_.notify_all();
    }
  }
  pdf_handle* h_;
  const ObjWriter& obj_;
  fs::path dir_;
  std::thread th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::pair<int, size_t>> queue_;
  bool busy_[2] = {false, false};
  bool done_ = false;
};

void print_values(const char* name, const double* tr, int first, int count) {
  std::cout << name << " ";
  for (int k = 0; k < count; ++k) std::cout << tr[first + k] << " ";
  std::cout << std::endl;
}

}  // namespace

int main(int argc, char* argv[]) {
  bool print_ac = false;
  const char* json = nullptr;
  for (int a = 1; a < argc; ++a) {
    const std::string arg = argv[a];
    if (arg == "--print-alart-curnier")
      print_ac = true;
    else if (!json)
      json = argv[a];
  }
  if (!json) {
    std::cerr << "Not enough arguments - 1 argument expected" << std::endl;
    std::cerr << " (1) Path of the json configuration file " << std::endl;
    return EXIT_FAILURE;
  }
  const fs::path scene_json_path(json);
  std::cout << "# Initializing." << std::endl;

  // output directory
  fs::path out_dir;
  unsigned number = 0;
  do {
    out_dir = fs::path("data" + std::to_string(number));
    ++number;
  } while (fs::is_directory(out_dir));
  fs::create_directories(out_dir);
  fs::copy_file(scene_json_path, out_dir / scene_json_path.filename());
  fs::create_directories(out_dir / "output");

  // scene, parameters, logs, simulation
  pdf_scene* scene = nullptr;
  check(pdf_scene_load_json(json, &scene), nullptr, "scene");
  pdf_params params;
  int32_t frames = 0, steps_per_frame = 0;
  check(pdf_params_load_json(json, &params, &frames, &steps_per_frame), nullptr, "parameters");
  params.trace_alart_curnier = print_ac ? 1 : 0;
  pdf_log* logs = nullptr;
  check(pdf_log_load_json(json, &logs), nullptr, "log");
  int32_t n_logs = 0;
  const pdf_log_entry* log_entries = nullptr;
  pdf_log_view(logs, &n_logs, &log_entries);
  pdf_scene_desc desc;
  check(pdf_scene_view(scene, &desc), nullptr, "scene view");
  if (desc.n_meshes < 1) die("the scene has no mesh");
  if (steps_per_frame < 1) die("\"Steps per frame\" must be at least 1");
  pdf_handle* sim = nullptr;
  check(pdf_create(&desc, &params, &sim), nullptr, "simulation");

  ObjWriter obj;
  const pdf_mesh_desc& m0 = desc.meshes[0];
  obj.v0 = m0.vertex_offset;
  obj.nv = m0.n_vertices;
  for (int t = m0.triangle_offset; t < m0.triangle_offset + m0.n_triangles; ++t)
    for (int c = 0; c < 3; ++c) obj.tris.push_back(desc.triangles[3 * t + c] - m0.vertex_offset);
  std::vector<std::vector<int32_t>> log_vertices(n_logs);
  for (int e = 0; e < n_logs; ++e)
    for (int k = 0; k < log_entries[e].n_vertices; ++k) {
      const int32_t i = log_entries[e].vertices[k];
      if (i < 0 || i >= m0.n_vertices) die("log vertex " + std::to_string(i) + " is not a vertex of mesh 0");
      log_vertices[e].push_back(m0.vertex_offset + i);
    }

  const size_t max_number_steps = (size_t)frames * (size_t)steps_per_frame;
  std::cout << "# Initialization done. Starting simulation, " << max_number_steps << " timesteps" << std::endl;
  std::list<int> milestones;
  for (int i = 5; i <= 100; i += 5) milestones.push_back(i);

  double current_time = 0.;
  std::vector<double> trace, gathered;
  {
    FrameWriter writer(sim, obj, out_dir / "output");
    int slot = 0;
    for (size_t i = 0; i < max_number_steps; ++i) {
      std::cout << "Time Step: " << i << std::endl;
      check(pdf_step(sim, 1, nullptr), sim, "step");
      if (print_ac) {
        int32_t iters = 0, nc = 0, ns = 0;
        check(pdf_get_alart_curnier_trace(sim, nullptr, 0, &iters, &nc, &ns), sim, "Alart-Curnier trace");
        trace.assign(2 * (size_t)iters * (nc + ns), 0.);
        check(pdf_get_alart_curnier_trace(sim, trace.data(), (int64_t)trace.size(), &iters, &nc, &ns), sim,
              "Alart-Curnier trace");
        std::vector<double> tang(nc + ns), norm(nc + ns);
        for (int it = 0; it < iters; ++it) {
          for (int k = 0; k < nc + ns; ++k) {
            tang[k] = trace[2 * ((size_t)it * (nc + ns) + k)];
            norm[k] = trace[2 * ((size_t)it * (nc + ns) + k) + 1];
          }
          if (nc > 0) {
            print_values("TangentialAlartCurnier", tang.data(), 0, nc);
            print_values("NormalAlartCurnier", norm.data(), 0, nc);
          }
          if (ns > 0) {
            print_values("SelfTangentialAlartCurnier", tang.data(), nc, ns);
            print_values("SelfNormalAlartCurnier", norm.data(), nc, ns);
          }
        }
      }
      current_time += params.time_step;
      std::cout << current_time << std::endl;
      for (int e = 0; e < n_logs; ++e) {
        const std::vector<int32_t>& vs = log_vertices[e];
        const bool pos = log_entries[e].kind == PDF_LOG_POSITION;
        gathered.assign(3 * vs.size(), 0.);
        if (!vs.empty())
          check(pdf_get_vertices(sim, vs.data(), (int32_t)vs.size(), pos ? gathered.data() : nullptr,
                                 pos ? nullptr : gathered.data()),
                sim, "log");
        std::cout << (pos ? "Position " : "Velocity ") << vs.size() << "\n";
        for (size_t k = 0; k < vs.size(); ++k) {
          std::cout << "v" << log_entries[e].vertices[k] << "\n";
          print_column(std::cout, gathered.data() + 3 * k);
          std::cout << "\n";
        }
      }
      if (i % (size_t)steps_per_frame == 0) {
        std::cout << "Saving Mesh" << std::endl;
        writer.submit(slot, i / (size_t)steps_per_frame);
        slot = 1 - slot;
      }
      if (!milestones.empty() && i >= milestones.front() * (max_number_steps - 1) / 100.) {
        std::cerr << milestones.front() << "% done" << std::endl;
        milestones.pop_front();
      }
    }
    writer.finish();
  }

  std::cout << "# Simulation done. Writing stats." << std::endl;
  check(pdf_export_stats(sim, (out_dir / "stats.txt").string().c_str()), sim, "stats");
  std::cout << "# Writing done. " << std::endl;
  pdf_destroy(sim);
  pdf_log_free(logs);
  pdf_scene_free(scene);
  return EXIT_SUCCESS;
}
