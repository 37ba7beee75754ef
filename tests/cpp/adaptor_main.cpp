// Drives the step loop through the C++ front of include/pdf_simulation.hpp
// the way the reference's main loop drives SimulationBase (src/main.cpp:40-124):
// scene and parameters from JSON, getSimulation, step(), exportStats().
//   adaptor_main scene.json steps positions.bin stats.txt
// Exit codes: 0 ok, 3 no usable CUDA device (PDF_NO_DEVICE), 1 other error.
#include <cstdio>
#include <cstdlib>
#include <fstream>

#include "pdf_simulation.hpp"

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s scene.json steps positions.bin stats.txt\n", argv[0]);
    return 1;
  }
  try {
    pdf::PhysicScene scene = pdf::getSceneFromJSONFileName(argv[1]);
    pdf::SimulationParameters params = pdf::getSimulationParametersFromJSONFileName(argv[1]);
    std::printf("scene: %d vertices, %d frames of %d steps, %d PD iterations\n", scene.getNumberOfVertices(),
                params.max_output_frame, params.sim_steps_per_frame, params.params.local_global_iterations);
    std::unique_ptr<pdf::SimulationGpu> simulation = pdf::getSimulation(scene, params);
    const int steps = std::atoi(argv[2]);
    for (int i = 0; i < steps; ++i) simulation->step();
    const std::vector<double> q = simulation->getGeneralizedPositions();
    std::ofstream out(argv[3], std::ios::binary);
    out.write(reinterpret_cast<const char*>(q.data()), (std::streamsize)(q.size() * sizeof(double)));
    std::ofstream of(argv[4]);
    simulation->exportStats(of);
    std::printf("stepped %d steps\n", steps);
  } catch (const pdf::Error& e) {
    std::printf("pdf error %d: %s\n", e.status(), e.what());
    return e.status() == PDF_NO_DEVICE ? 3 : 1;
  }
  return 0;
}
