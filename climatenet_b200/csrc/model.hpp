// model.hpp — host-side set-up of one cloth scene for the device step loop.
//
// Builds, from a pdf_scene_desc, everything the reference computes once in
// its constructors: mesh topology (src/geometry/Mesh.cpp:31-56, 219-292),
// lumped masses (src/physics/PhysicMesh.cpp:115-151), the spring / bending /
// attachment constraint rows of A (SpringConstraint.cpp:42-54,
// BendingConstraint.cpp:47-104, AttachmentConstraint.cpp:31-42), A^T A and the
// global-step matrix M + dt^2 A^T A (SimulationSpeed.cpp:230-236).
//
// The constraint data is laid out vertex-centric for the device local step:
// vertex i gathers its spring terms and the bending rows it belongs to from its
// 1-ring instead of scattering constraint contributions with atomics.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/pdf.h"

namespace pdfb {

struct Model {
  int N = 0;                      // vertices
  int n_rows = 0;                 // rows(A)
  int64_t nnz_a = 0;
  std::vector<double> rest;       // 3N
  std::vector<double> q0, v0;     // 3N initial state
  std::vector<double> mass;       // N
  std::vector<int> vmesh;         // containing mesh per vertex
  std::vector<int> tris;          // 3T scene-global
  std::vector<pdf_mesh_desc> meshes;

  // 1-ring adjacency (CSR over vertices, sorted by neighbour index)
  std::vector<int> ring_ptr, ring_idx;
  // per ring slot: spring coefficient kappa_ij = sqrt(k) * (sqrt(k) * L_ij)
  // (A entry times projection scale), and the coefficient of vertex i in the
  // bending row of neighbour j (0 when j is on the border).
  std::vector<double> ring_kappa, ring_bend;
  // own bending row (or -1) and the coefficient of i in it
  std::vector<int> bend_of;       // N
  std::vector<double> self_bend;  // N
  // bending constraints: centre + clockwise ring, unweighted mean-value
  // coefficients, weight sqrt(b), rest norm
  std::vector<int> bend_ptr, bend_idx;
  std::vector<double> bend_coef, bend_w, bend_rest;
  // attachment term sum_pins sqrt(w) * (sqrt(w) x0) per vertex (3N), constant
  std::vector<double> pin_term;
  // per vertex: the stiffness of its springs (the weight sqrt(k) squared, the
  // same for every spring of a mesh) and the summed weight of its pins; with
  // them the local step forms the residual in force form (FP32 mode)
  std::vector<double> spring_k, pin_w;
  bool has_pins = false;

  // A^T A in CSR (full symmetric), sorted columns
  std::vector<int> ata_ptr, ata_col;
  std::vector<double> ata_val;

  // obstacles & friction
  std::vector<pdf_obstacle> obstacles;
  std::vector<std::vector<double>> obstacle_vertices;
  std::vector<std::vector<int>> obstacle_triangles;
  int n_materials = 0;
  std::vector<double> friction;

  // per-mesh clockwise rings are needed only for bending; the 1-ring above is
  // what self-collision pairing uses.
};

// Throws std::invalid_argument on malformed input.
void build_model(const pdf_scene_desc& sc, const pdf_params& p, Model& m);

}  // namespace pdfb
