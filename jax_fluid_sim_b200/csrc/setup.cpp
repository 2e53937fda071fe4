// Host-side geometry metrics for building a plan: the isoparametric map's Jacobian, its
// determinant and inverse at a set of reference points, and the face normals and area weights
// derived from it (the reference forms the same quantities with dense einsums,
// hybrid/geometry.py:139-203 for elements and :299-353 for faces).
//
// These are O(elements x points) loops over small 3x3 matrices; they run on the host cores in
// threads, one contiguous range of elements per thread, each element's sums in a fixed order.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "dgb200.h"

namespace dgb {
int set_error(int code, const char* msg);   // defined with the plan code
}

namespace {

template <typename Body>
void parallel_ranges(int count, Body body) {
  const int hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = std::max(1, std::min(hw, count / 256));
  if (nt <= 1) {
    body(0, count);
    return;
  }
  std::vector<std::thread> pool;
  const int step = (count + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const int lo = t * step, hi = std::min(count, lo + step);
    if (lo < hi) pool.emplace_back(body, lo, hi);
  }
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" int dgb_map_metrics(const double* nodes, const int32_t* index, int count, int num_nodes,
                               const double* grad, int num_points, const double* weights, const double* tangents,
                               const double* orientation, double* jacobian, double* det, double* inv_jacobian,
                               double* wdet, double* normals, double* area_weights) {
  if (count < 0 || num_nodes < 1 || num_points < 1 || !nodes || !grad)
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad map-metrics sizes or null nodes/gradients");
  if ((wdet || area_weights) && !weights) return dgb::set_error(DGB_ERR_ARGUMENT, "wdet and area weights need weights");
  if ((normals || area_weights) && (!tangents || !orientation))
    return dgb::set_error(DGB_ERR_ARGUMENT, "normals need tangents and an orientation");
  const int n = num_nodes, Q = num_points;
  parallel_ranges(count, [=](int lo, int hi) {
    for (int i = lo; i < hi; ++i) {
      const double* x = nodes + (size_t)(index ? index[i] : i) * n * 3;
      for (int q = 0; q < Q; ++q) {
        const double* g = grad + (size_t)q * n * 3;
        double J[3][3] = {};
        for (int k = 0; k < n; ++k)
          for (int d = 0; d < 3; ++d)
            for (int r = 0; r < 3; ++r) J[d][r] += x[k * 3 + d] * g[k * 3 + r];
        const size_t o = (size_t)i * Q + q;
        if (jacobian)
          for (int t = 0; t < 9; ++t) jacobian[o * 9 + t] = J[t / 3][t % 3];
        const double A = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double B = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const double C = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        const double D = J[0][0] * A + J[0][1] * B + J[0][2] * C;
        if (det) det[o] = D;
        if (wdet) wdet[o] = weights[q] * std::fabs(D);
        if (inv_jacobian) {
          const double s = 1.0 / D;
          double* v = inv_jacobian + o * 9;
          v[0] = A * s;
          v[1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * s;
          v[2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * s;
          v[3] = B * s;
          v[4] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * s;
          v[5] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * s;
          v[6] = C * s;
          v[7] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * s;
          v[8] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * s;
        }
        if (normals || area_weights) {
          // physical tangents J t_u, J t_v; their cross product, oriented along the face's
          // owner-to-neighbour direction, gives the unit normal and the area element
          const double* tu = tangents + (size_t)q * 6;
          const double* tv = tu + 3;
          double a[3], b[3];
          for (int d = 0; d < 3; ++d) {
            a[d] = J[d][0] * tu[0] + J[d][1] * tu[1] + J[d][2] * tu[2];
            b[d] = J[d][0] * tv[0] + J[d][1] * tv[1] + J[d][2] * tv[2];
          }
          double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
          const double* h = orientation + (size_t)i * 3;
          const double sgn = (c[0] * h[0] + c[1] * h[1] + c[2] * h[2]) >= 0.0 ? 1.0 : -1.0;
          for (double& v : c) v *= sgn;
          const double mag = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
          if (normals)
            for (int d = 0; d < 3; ++d) normals[o * 3 + d] = c[d] / mag;
          if (area_weights) area_weights[o] = weights[q] * mag;
        }
      }
    }
  });
  return DGB_OK;
}

// Subcell face metrics of the MOOD subcell plan (hybrid/subcell.py:336-360), per element: the area
// vector of each subcell face (a triangle p0 p1 p2 gives (p1 - p0) x (p2 - p0) / 2, a quadrilateral
// adds (p2 - p0) x (p3 - p0) / 2), turned to point from the owner subcell's centre toward the
// neighbour's (or, without a neighbour, toward the face centre), its length and unit vector, and
// the face centre (the mean of its vertices).
extern "C" int dgb_subcell_face_metrics(const double* vertices, int count, int num_vertices, const int32_t* faces,
                                        const int32_t* face_sizes, int num_faces, const double* centers,
                                        int num_subcells, const int32_t* owners, const int32_t* neighbors,
                                        double* normals, double* areas, double* face_centers) {
  if (count < 0 || num_vertices < 1 || num_faces < 0 || num_subcells < 1 || !vertices || !faces || !face_sizes ||
      !centers || !owners || !normals || !areas)
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad subcell face-metrics argument");
  for (int f = 0; f < num_faces; ++f) {
    if (face_sizes[f] != 3 && face_sizes[f] != 4) return dgb::set_error(DGB_ERR_ARGUMENT, "faces have 3 or 4 vertices");
    for (int k = 0; k < face_sizes[f]; ++k)
      if (faces[f * 4 + k] < 0 || faces[f * 4 + k] >= num_vertices)
        return dgb::set_error(DGB_ERR_ARGUMENT, "face vertex out of range");
    if (owners[f] < 0 || owners[f] >= num_subcells || (neighbors && (neighbors[f] < 0 || neighbors[f] >= num_subcells)))
      return dgb::set_error(DGB_ERR_ARGUMENT, "face subcell out of range");
  }
  const int V = num_vertices, F = num_faces, S = num_subcells;
  parallel_ranges(count, [=](int lo, int hi) {
    for (int e = lo; e < hi; ++e) {
      const double* pv = vertices + (size_t)e * V * 3;
      const double* cen = centers + (size_t)e * S * 3;
      for (int f = 0; f < F; ++f) {
        const int n = face_sizes[f];
        const double* p[4];
        for (int k = 0; k < n; ++k) p[k] = pv + faces[f * 4 + k] * 3;
        double u[3], w[3], a[3], fc[3];
        for (int d = 0; d < 3; ++d) {
          u[d] = p[1][d] - p[0][d];
          w[d] = p[2][d] - p[0][d];
        }
        a[0] = 0.5 * (u[1] * w[2] - u[2] * w[1]);
        a[1] = 0.5 * (u[2] * w[0] - u[0] * w[2]);
        a[2] = 0.5 * (u[0] * w[1] - u[1] * w[0]);
        if (n == 4) {
          double z[3];
          for (int d = 0; d < 3; ++d) z[d] = p[3][d] - p[0][d];
          a[0] = a[0] + 0.5 * (w[1] * z[2] - w[2] * z[1]);
          a[1] = a[1] + 0.5 * (w[2] * z[0] - w[0] * z[2]);
          a[2] = a[2] + 0.5 * (w[0] * z[1] - w[1] * z[0]);
        }
        for (int d = 0; d < 3; ++d) {
          double s = p[0][d] + p[1][d];
          for (int k = 2; k < n; ++k) s += p[k][d];
          fc[d] = s / n;
        }
        const double* oc = cen + owners[f] * 3;
        double dir[3];
        for (int d = 0; d < 3; ++d) dir[d] = neighbors ? cen[neighbors[f] * 3 + d] - oc[d] : fc[d] - oc[d];
        const double sgn = (a[0] * dir[0] + a[1] * dir[1] + a[2] * dir[2]) >= 0.0 ? 1.0 : -1.0;
        for (double& v : a) v *= sgn;
        const double mag = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        const size_t o = (size_t)e * F + f;
        for (int d = 0; d < 3; ++d) normals[o * 3 + d] = a[d] / mag;
        areas[o] = mag;
        if (face_centers)
          for (int d = 0; d < 3; ++d) face_centers[o * 3 + d] = fc[d];
      }
    }
  });
  return DGB_OK;
}

// Affine test of a block's per-point inverse Jacobians jinv [count][num_points][9]: an element is
// affine when every point's entries equal the first point's to tol relative to the element's
// largest |entry|; mean[count][9] receives the mean over the points (summed in point order).
extern "C" int dgb_affine_test(const double* jinv, int count, int num_points, double tol, uint8_t* affine,
                               double* mean) {
  if (count < 0 || num_points < 1 || !jinv || !affine || !mean)
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad affine-test argument");
  const int Q = num_points;
  parallel_ranges(count, [=](int lo, int hi) {
    for (int e = lo; e < hi; ++e) {
      const double* J = jinv + (size_t)e * Q * 9;
      double dev = 0.0, big = 0.0, s[9] = {};
      for (int q = 0; q < Q; ++q)
        for (int k = 0; k < 9; ++k) {
          const double v = J[q * 9 + k];
          dev = std::max(dev, std::fabs(v - J[k]));
          big = std::max(big, std::fabs(v));
          s[k] += v;
        }
      affine[e] = dev / std::max(big, 1e-300) <= tol ? 1 : 0;
      for (int k = 0; k < 9; ++k) mean[(size_t)e * 9 + k] = s[k] / Q;
    }
  });
  return DGB_OK;
}
