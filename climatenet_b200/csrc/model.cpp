// model.cpp — host-side scene set-up (topology, masses, constraint tables,
// A^T A).  See model.hpp.
#include "model.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace pdfb {
namespace {

struct P3 {
  double x, y, z;
};
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double dot3(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len3(P3 a) { return std::sqrt(dot3(a, a)); }
inline P3 crs(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline P3 at3(const std::vector<double>& v, int i) { return {v[3 * (size_t)i], v[3 * (size_t)i + 1], v[3 * (size_t)i + 2]}; }

// tan(half angle at v2 of the triangle v1 v2 v3), written (1 - cos) / sin as in
// getMeanValue (src/geometry/geometry_util.cpp:766-775).
double half_angle_tan(P3 v1, P3 v2, P3 v3) {
  P3 e1 = sub(v1, v2), e2 = sub(v3, v2);
  double l = len3(e1) * len3(e2);
  double cosv = dot3(e1, e2) / l;
  double num = 1 - cosv;
  if (num == 0) return 0;
  return num / (len3(crs(e1, e2)) / l);
}

// Halfedge topology of one mesh: directed halfedge 3f+i runs
// tris[f][i] -> tris[f][(i+1)%3].  Opposites are found by sorting.
struct HalfEdges {
  std::vector<int> opp;  // opposite halfedge or -1
};

void build_halfedges(const std::vector<int>& tris, int t0, int t1, HalfEdges& he) {
  const int nh = 3 * (t1 - t0);
  std::vector<std::pair<uint64_t, int>> keys(nh);
  for (int f = t0; f < t1; ++f)
    for (int i = 0; i < 3; ++i) {
      uint32_t a = (uint32_t)tris[3 * (size_t)f + i], b = (uint32_t)tris[3 * (size_t)f + (i + 1) % 3];
      keys[3 * (f - t0) + i] = {((uint64_t)a << 32) | b, 3 * (f - t0) + i};
    }
  std::vector<std::pair<uint64_t, int>> sorted = keys;
  std::sort(sorted.begin(), sorted.end());
  he.opp.assign(nh, -1);
  for (int h = 0; h < nh; ++h) {
    uint64_t k = keys[h].first;
    uint64_t rk = (k << 32) | (k >> 32);
    auto it = std::lower_bound(sorted.begin(), sorted.end(), std::make_pair(rk, -1));
    if (it != sorted.end() && it->first == rk) he.opp[h] = it->second;
  }
}

}  // namespace

void build_model(const pdf_scene_desc& sc, const pdf_params& p, Model& m) {
  if (sc.n_vertices <= 0 || !sc.rest_positions) throw std::invalid_argument("scene has no vertices");
  if (sc.n_meshes <= 0 || !sc.meshes) throw std::invalid_argument("scene has no dynamic mesh");
  if (sc.n_triangles <= 0 || !sc.triangles) throw std::invalid_argument("scene has no triangles");
  if (sc.n_materials <= 0 || !sc.friction) throw std::invalid_argument("missing friction table");
  if (!(p.time_step > 0.) || !std::isfinite(p.time_step)) throw std::invalid_argument("time step must be positive");
  if (p.local_global_iterations <= 0) throw std::invalid_argument("LocalGlobal must be positive");
  const int N = sc.n_vertices;
  m.N = N;
  m.rest.assign(sc.rest_positions, sc.rest_positions + 3 * (size_t)N);
  m.q0 = sc.positions ? std::vector<double>(sc.positions, sc.positions + 3 * (size_t)N) : m.rest;
  m.v0 = sc.velocities ? std::vector<double>(sc.velocities, sc.velocities + 3 * (size_t)N)
                       : std::vector<double>(3 * (size_t)N, 0.);
  for (size_t d = 0; d < m.q0.size(); ++d)
    if (!std::isfinite(m.q0[d]) || !std::isfinite(m.v0[d]) || !std::isfinite(m.rest[d]))
      throw std::invalid_argument("non-finite position or velocity in the scene");
  m.tris.assign(sc.triangles, sc.triangles + 3 * (size_t)sc.n_triangles);
  for (int x : m.tris)
    if (x < 0 || x >= N) throw std::invalid_argument("triangle index out of range");
  m.meshes.assign(sc.meshes, sc.meshes + sc.n_meshes);
  m.n_materials = sc.n_materials;
  m.friction.assign(sc.friction, sc.friction + (size_t)sc.n_materials * sc.n_materials);
  m.vmesh.assign(N, -1);
  m.mass.assign(N, 0.);
  m.bend_of.assign(N, -1);
  m.self_bend.assign(N, 0.);
  m.pin_term.assign(3 * (size_t)N, 0.);
  m.spring_k.assign(N, 0.);
  m.pin_w.assign(N, 0.);

  // A rows: (vertex, value) lists, in the reference's row order: per mesh the
  // springs (edge creation order) then the bending rows (vertex order), then
  // the attachment rows.
  std::vector<int> row_ptr{0};
  std::vector<int> row_v;
  std::vector<double> row_a;
  auto push_row = [&](std::initializer_list<std::pair<int, double>> e) {
    for (auto& x : e) {
      row_v.push_back(x.first);
      row_a.push_back(x.second);
    }
    row_ptr.push_back((int)row_v.size());
  };

  std::vector<std::vector<std::pair<int, double>>> nb(N);  // (j, kappa)

  for (int mi = 0; mi < sc.n_meshes; ++mi) {
    const pdf_mesh_desc& md = sc.meshes[mi];
    if (md.vertex_offset < 0 || md.n_vertices <= 0 || md.vertex_offset + md.n_vertices > N ||
        md.triangle_offset < 0 || md.n_triangles <= 0 || md.triangle_offset + md.n_triangles > sc.n_triangles)
      throw std::invalid_argument("mesh ranges out of bounds");
    if (md.material < 0 || md.material >= sc.n_materials) throw std::invalid_argument("mesh material out of range");
    // A negative stiffness is not rejected here: like the reference, it makes
    // the global-step matrix indefinite and the factorisation reports it.
    if (!(md.area_density > 0.)) throw std::invalid_argument("area density must be positive");
    const int v0 = md.vertex_offset, v1 = v0 + md.n_vertices;
    const int t0 = md.triangle_offset, t1 = t0 + md.n_triangles;
    for (int v = v0; v < v1; ++v) {
      if (m.vmesh[v] != -1) throw std::invalid_argument("meshes overlap");
      m.vmesh[v] = mi;
    }
    for (int f = t0; f < t1; ++f)
      for (int k = 0; k < 3; ++k) {
        int x = m.tris[3 * (size_t)f + k];
        if (x < v0 || x >= v1) throw std::invalid_argument("triangle uses a vertex of another mesh");
      }
    HalfEdges he;
    build_halfedges(m.tris, t0, t1, he);
    const int nh = 3 * (t1 - t0);
    auto hsrc = [&](int h) { return m.tris[3 * (size_t)(t0 + h / 3) + h % 3]; };
    auto htgt = [&](int h) { return m.tris[3 * (size_t)(t0 + h / 3) + (h % 3 + 1) % 3]; };
    auto hnext = [&](int h) { return 3 * (h / 3) + (h % 3 + 1) % 3; };
    std::vector<char> border(N, 0), has_face(N, 0);
    std::vector<int> in_he(N, -1);  // one incoming halfedge per vertex
    for (int h = 0; h < nh; ++h) {
      has_face[hsrc(h)] = 1;
      if (in_he[htgt(h)] < 0) in_he[htgt(h)] = h;
      if (he.opp[h] < 0) {
        border[hsrc(h)] = 1;
        border[htgt(h)] = 1;
      }
    }
    // lumped masses: rho * area / 3 summed over incident faces
    for (int f = t0; f < t1; ++f) {
      P3 a = at3(m.rest, m.tris[3 * (size_t)f]), b = at3(m.rest, m.tris[3 * (size_t)f + 1]),
         c = at3(m.rest, m.tris[3 * (size_t)f + 2]);
      P3 cr = crs(sub(b, a), sub(c, a));
      double area = std::sqrt(dot3(cr, cr) / 4);
      for (int k = 0; k < 3; ++k) m.mass[m.tris[3 * (size_t)f + k]] += md.area_density * area;
    }
    for (int v = v0; v < v1; ++v) m.mass[v] /= 3;
    // springs, one per undirected edge in order of first appearance
    const double sk = std::sqrt(md.stretching);
    for (int v = v0; v < v1; ++v) m.spring_k[v] = sk * sk;
    for (int h = 0; h < nh; ++h) {
      int o = he.opp[h];
      if (o >= 0 && o < h) continue;  // edge already created by its opposite
      int a = htgt(h), b = hsrc(h);
      double L = len3(sub(at3(m.rest, a), at3(m.rest, b)));
      push_row({{a, sk}, {b, -sk}});
      double kappa = sk * (sk * L);
      nb[a].push_back({b, kappa});
      nb[b].push_back({a, kappa});
    }
    // bending rows for interior vertices, clockwise 1-ring (h -> opposite(next(h)))
    const double sb = std::sqrt(md.bending);
    for (int v = v0; v < v1; ++v) {
      if (border[v] || !has_face[v] || in_he[v] < 0) continue;
      std::vector<int> ring;
      int h = in_he[v], h0 = h, guard = 0;
      bool ok = true;
      do {
        ring.push_back(hsrc(h));
        int o = he.opp[hnext(h)];
        if (o < 0) {
          ok = false;
          break;
        }
        h = o;
      } while (h != h0 && ++guard < 4096);
      if (!ok || ring.size() < 3) continue;
      const size_t n = ring.size();
      P3 mid = at3(m.rest, v);
      std::vector<double> coef(n + 1, 0.);
      for (size_t i = 0; i < n; ++i) {
        P3 vx = at3(m.rest, ring[i]), cw = at3(m.rest, ring[(i + 1) % n]), ccw = at3(m.rest, ring[(i + n - 1) % n]);
        double c = (half_angle_tan(vx, mid, cw) + half_angle_tan(vx, ccw, mid)) / len3(sub(vx, mid));
        coef[0] += c;
        coef[i + 1] = -c;
      }
      const int b = (int)m.bend_w.size();
      m.bend_of[v] = b;
      if (m.bend_ptr.empty()) m.bend_ptr.push_back(0);
      m.bend_idx.push_back(v);
      m.bend_coef.push_back(coef[0]);
      for (size_t i = 0; i < n; ++i) {
        m.bend_idx.push_back(ring[i]);
        m.bend_coef.push_back(coef[i + 1]);
      }
      m.bend_ptr.push_back((int)m.bend_idx.size());
      double rx = 0, ry = 0, rz = 0;
      for (size_t k = 0; k <= n; ++k) {
        P3 x = at3(m.rest, k == 0 ? v : ring[k - 1]);
        rx += coef[k] * x.x;
        ry += coef[k] * x.y;
        rz += coef[k] * x.z;
      }
      m.bend_rest.push_back(std::sqrt(rx * rx + ry * ry + rz * rz));
      m.bend_w.push_back(sb);
      row_v.push_back(v);
      row_a.push_back(sb * coef[0]);
      for (size_t i = 0; i < n; ++i) {
        row_v.push_back(ring[i]);
        row_a.push_back(sb * coef[i + 1]);
      }
      row_ptr.push_back((int)row_v.size());
    }
  }
  for (int v = 0; v < N; ++v) {
    if (m.vmesh[v] < 0) throw std::invalid_argument("vertex not covered by any mesh");
    if (!(m.mass[v] > 0.)) throw std::invalid_argument("vertex with zero mass (not on any triangle)");
  }
  if (m.bend_ptr.empty()) m.bend_ptr.push_back(0);
  // attachment rows
  for (int k = 0; k < sc.n_pins; ++k) {
    int v = sc.pin_vertices[k];
    double w = sc.pin_weights[k];
    if (v < 0 || v >= N || !(w >= 0.)) throw std::invalid_argument("invalid attachment");
    double sw = std::sqrt(w);
    push_row({{v, sw}});
    for (int c = 0; c < 3; ++c) m.pin_term[3 * (size_t)v + c] += sw * (sw * sc.pin_positions[3 * (size_t)k + c]);
    m.pin_w[v] += sw * sw;
    m.has_pins = true;
  }
  m.n_rows = (int)row_ptr.size() - 1;
  m.nnz_a = (int64_t)row_v.size();

  // 1-ring tables (sorted by neighbour) with spring and bending coefficients
  m.ring_ptr.assign(N + 1, 0);
  for (int v = 0; v < N; ++v) {
    std::sort(nb[v].begin(), nb[v].end());
    m.ring_ptr[v + 1] = m.ring_ptr[v] + (int)nb[v].size();
  }
  m.ring_idx.resize(m.ring_ptr[N]);
  m.ring_kappa.resize(m.ring_ptr[N]);
  m.ring_bend.assign(m.ring_ptr[N], 0.);
  for (int v = 0; v < N; ++v)
    for (int k = 0; k < (int)nb[v].size(); ++k) {
      m.ring_idx[m.ring_ptr[v] + k] = nb[v][k].first;
      m.ring_kappa[m.ring_ptr[v] + k] = nb[v][k].second;
    }
  for (int b = 0; b + 1 < (int)m.bend_ptr.size(); ++b) {
    const int c = m.bend_idx[m.bend_ptr[b]];
    m.self_bend[c] = m.bend_w[b] * m.bend_coef[m.bend_ptr[b]];
    for (int k = m.bend_ptr[b] + 1; k < m.bend_ptr[b + 1]; ++k) {
      const int i = m.bend_idx[k];  // vertex i is in the row of centre c
      auto beg = m.ring_idx.begin() + m.ring_ptr[i], end = m.ring_idx.begin() + m.ring_ptr[i + 1];
      auto it = std::lower_bound(beg, end, c);
      if (it == end || *it != c) throw std::logic_error("bending ring neighbour is not a mesh neighbour");
      m.ring_bend[m.ring_ptr[i] + (it - m.ring_idx.begin() - m.ring_ptr[i])] = m.bend_w[b] * m.bend_coef[k];
    }
  }

  // A^T A: row i = sum over rows r containing i of A[r,i] * A[r,:]
  std::vector<std::vector<std::pair<int, int>>> vrows(N);  // (row, position in row)
  for (int r = 0; r < m.n_rows; ++r)
    for (int k = row_ptr[r]; k < row_ptr[r + 1]; ++k) vrows[row_v[k]].push_back({r, k});
  std::vector<std::vector<int>> cols(N);
  std::vector<std::vector<double>> vals(N);
#pragma omp parallel
  {
    std::vector<double> acc(N, 0.);
    std::vector<int> mark(N, -1), list;
#pragma omp for schedule(dynamic, 512)
    for (int i = 0; i < N; ++i) {
      list.clear();
      for (auto& rk : vrows[i]) {
        const double ai = row_a[rk.second];
        for (int k = row_ptr[rk.first]; k < row_ptr[rk.first + 1]; ++k) {
          const int j = row_v[k];
          if (mark[j] != i) {
            mark[j] = i;
            acc[j] = 0.;
            list.push_back(j);
          }
          acc[j] += ai * row_a[k];
        }
      }
      std::sort(list.begin(), list.end());
      cols[i] = list;
      vals[i].resize(list.size());
      for (size_t k = 0; k < list.size(); ++k) vals[i][k] = acc[list[k]];
    }
  }
  m.ata_ptr.assign(N + 1, 0);
  for (int i = 0; i < N; ++i) m.ata_ptr[i + 1] = m.ata_ptr[i] + (int)cols[i].size();
  m.ata_col.resize(m.ata_ptr[N]);
  m.ata_val.resize(m.ata_ptr[N]);
  for (int i = 0; i < N; ++i) {
    std::copy(cols[i].begin(), cols[i].end(), m.ata_col.begin() + m.ata_ptr[i]);
    std::copy(vals[i].begin(), vals[i].end(), m.ata_val.begin() + m.ata_ptr[i]);
  }
  // every vertex must at least carry its diagonal (mass) entry
  for (int i = 0; i < N; ++i) {
    bool diag = false;
    for (int k = m.ata_ptr[i]; k < m.ata_ptr[i + 1]; ++k) diag |= (m.ata_col[k] == i);
    if (!diag) throw std::invalid_argument("vertex without any constraint (isolated vertex)");
  }

  // obstacles
  for (int k = 0; k < sc.n_obstacles; ++k) {
    pdf_obstacle o = sc.obstacles[k];
    if (o.type < 0 || o.type > 5) throw std::invalid_argument("unknown obstacle type");
    if (o.type == PDF_OBSTACLE_BOX && !(o.size[0] >= 0. && o.size[1] >= 0. && o.size[2] >= 0.))
      throw std::invalid_argument("box obstacle with a negative size");
    if (o.material < 0 || o.material >= sc.n_materials) throw std::invalid_argument("obstacle material out of range");
    std::vector<double> ov;
    std::vector<int> ot;
    if (o.type == PDF_OBSTACLE_MOVING_MESH && (o.n_frames < 2 || !(o.frame_interval > 0.)))
      throw std::invalid_argument("moving mesh needs at least two key frames and a positive interval");
    if (o.type == PDF_OBSTACLE_MESH || o.type == PDF_OBSTACLE_MOVING_MESH) {
      if (o.n_vertices <= 0 || o.n_triangles <= 0 || !o.vertices || !o.triangles)
        throw std::invalid_argument("mesh obstacle without geometry");
      const size_t frames = o.type == PDF_OBSTACLE_MOVING_MESH ? (size_t)o.n_frames : 1;
      ov.assign(o.vertices, o.vertices + 3 * (size_t)o.n_vertices * frames);
      ot.assign(o.triangles, o.triangles + 3 * (size_t)o.n_triangles);
      for (int x : ot)
        if (x < 0 || x >= o.n_vertices) throw std::invalid_argument("mesh obstacle index out of range");
    }
    o.vertices = nullptr;
    o.triangles = nullptr;
    m.obstacles.push_back(o);
    m.obstacle_vertices.push_back(std::move(ov));
    m.obstacle_triangles.push_back(std::move(ot));
  }
}

}  // namespace pdfb
