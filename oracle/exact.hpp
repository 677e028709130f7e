// Oracle exact signed distance of a B-rep solid and its brick-cache bake (f64).
// Restates crates/icam-core/src/solid3.rs (Solid3, BoxTree, Exact), surface3.rs
// (analytic feet, NurbsSurf::closest_trimmed), curve3.rs (Edge3, Spline3) and
// crates/icam-sim/src/partcache.rs (decide, exact_brick, packed).
// TEST INFRASTRUCTURE ONLY.
#pragma once

#include <memory>
#include <string>

#include "../include/icam_solid.h"
#include "geom.hpp"
#include "trim.hpp"

namespace oracle {

enum SurfKind { PLANE = 0, CYLINDER = 1, CONE = 2, SPHERE = 3, TORUS = 4, NURBS = 5 };

// surface3.rs:1197-1204 SurfHit
struct SurfHit {
  V3 q;
  double dist;
  double u, v;
  V3 n;
};

// A rational B-spline surface as its grid of Bezier spans and a quadtree over them
// (surface3.rs:1110-1160, build 1093-1133).
struct NurbsSurf {
  int du = 0, dv = 0, nsu = 0, nsv = 0;
  std::vector<Patch> spans;  // (a, b) at a * nsv + b
  std::vector<double> ub, vb;
  struct QNode {
    Box box;
    int i0, i1, j0, j1;
    std::vector<int> kids;
  };
  std::vector<QNode> nodes;
  // surface3.rs:579-591 Creases: the domain sides the surface collapses on to one point
  // (u held at each of cu, v at each of cv); a patch with a side on one is never cleared
  // by the critical-point test
  std::vector<double> cu, cv;
  bool touches(const Patch& pa) const;
  void build_tree();
  int build(int i0, int i1, int j0, int j1);
  const Patch& span(int a, int b) const { return spans[a * nsv + b]; }
  Box bbox() const { return nodes[0].box; }
  SEval eval(double u, double v) const;
  // surface3.rs:1214-1297 closest_trimmed; returns (hit?, complete, pops)
  bool closest_trimmed(V3 p, double cutoff, const Trim2* trim, SurfHit* hit, bool* complete, int* pops) const;
  // surface3.rs:1314-1366 descend
  bool descend(V3 p, double u, double v, bool border, SurfHit* hit) const;
  // surface3.rs:1444-1499 closest
  bool closest(V3 p, double cutoff, SurfHit* hit) const;
  int span_of(const std::vector<double>& br, double x) const;
};

struct Surf {
  int kind = PLANE;
  Frame f;
  double a = 0, b = 0;  // r / (r, semi-angle) / r / (major, minor)
  std::shared_ptr<NurbsSurf> ns;
  V3 foot(V3 p) const;
  V3 normal(V3 x) const;
  void uv(V3 q, double* u, double* v) const;
};

// curve3.rs:545-565 Foot3
enum Near { INTERIOR = 0, START = 1, END = 2 };
struct Foot3 {
  V3 q;
  double dist;
  double t;
  int near;
  V3 tangent;
};

// curve3.rs:336-372 Spline3: flat rational Bezier pieces
struct Spline3 {
  std::vector<Bez3> pieces;
  std::vector<double> thick;
  std::vector<Box> boxes;
  bool closest(V3 p, double cutoff, Foot3* out) const;
};

// curve3.rs:489-498 Edge3
struct Edge3 {
  int kind = 0;  // 0 line, 1 arc, 2 spline
  V3 a, b;
  Frame f;
  double r = 0, t0 = 0, sweep = 0;
  std::shared_ptr<Spline3> sp;
  V3 at(double s) const;
  Foot3 closest(V3 p) const;
  bool closest_below(V3 p, double cutoff, Foot3* out) const;
  V3 tangent_at(double s) const;
  Box bbox() const;
};

struct Face {
  Surf surf;
  double sense = 1;
  Trim2 trim;
  std::vector<std::vector<std::pair<int, bool>>> loops;  // (edge, rev)
  V3 normal(V3 x) const { return surf.normal(x) * sense; }
};

struct EdgeRec {
  Edge3 curve;
  int faces[2];
  int v[2];
  Box box;
};

struct Vert {
  V3 p, pn;
};

// solid3.rs:314-321 Sd, Feature
struct Sd {
  double d;
  V3 q;
  int kind;  // 0 face, 1 edge, 2 vertex
  int id;
  bool unsure;
};

// solid3.rs:1570-1583 ExactStats
struct ExactStats {
  int pops = 0;
  bool capped = false;
  bool cusp = false;
  int features = 0;
};

// solid3.rs:97-236 BoxTree
class BoxTree {
 public:
  void init(const std::vector<Box>& boxes);
  template <class F>
  void visit(const Box& q, double d, F&& f) const {
    if (!nodes_.empty()) visit_at(0, q, d, f);
  }
  template <class F>
  void nearest_first(V3 p, double bound, F&& f) const;
  Box boxes_of(size_t id) const { return boxes_[at_[id]]; }

 private:
  std::vector<Box> boxes_;
  std::vector<size_t> ids_, at_;
  struct Node {
    Box b;
    size_t a, e;
  };
  std::vector<Node> nodes_;
  Box build(size_t k, size_t a, size_t b);
  template <class F>
  void visit_at(size_t k, const Box& q, double d, F& f) const {
    const Node& n = nodes_[k];
    if (box_gap(n.b, q) > d) return;
    if (n.e - n.a <= 4) {
      for (size_t i = n.a; i < n.e; i++)
        if (box_gap(boxes_[i], q) <= d) f(ids_[i]);
      return;
    }
    visit_at(2 * k + 1, q, d, f);
    visit_at(2 * k + 2, q, d, f);
  }
};

// solid3.rs:1562-1568 C0Line: an interior knot line of a B-spline face where the surface
// is only C0 (a crease): the direction held fixed (0: u), its value, and per span of the
// other direction the line's piece (parameter along the line) with the spans before and
// after it. Found here from the surface's geometry (the spans' normals differ across the
// line), where the reference takes the knots of full multiplicity: a knot line across
// which the normal is continuous needs no line of its own (its nearest points are
// critical points of the spans on either side).
struct C0Line {
  int face = 0;
  int k = 0;
  double value = 0;
  std::vector<Bez3> pieces;
  std::vector<const Patch*> before, after;
};

// solid3.rs:1551-1553 a pole: the point a B-spline face's side collapses on to, inside
// the face and at no vertex, with the fan pseudo-normal (times the face's sense)
struct Pole {
  int face = 0;
  V3 x, n;
};

class Exact {
 public:
  bool init(const IcamSolidDesc* d, std::string* err);
  // solid3.rs:1750-1816
  Sd sdf_within(V3 p, double bound, ExactStats* st) const;
  Sd sdf(V3 p, ExactStats* st) const { return sdf_within(p, INF, st); }
  // solid3.rs:1661-1690
  std::vector<size_t> candidates(V3 c, double r, double d) const;
  int kind_of(size_t id) const;
  size_t nf() const { return faces.size(); }
  size_t ne() const { return edges.size(); }
  size_t nv() const { return verts.size(); }
  double tol = 1e-9;
  std::vector<Face> faces;
  std::vector<EdgeRec> edges;
  std::vector<Vert> verts;
  std::vector<C0Line> lines;  // the tree's ids after the vertices
  std::vector<Pole> poles;    // the tree's ids after the knot lines
  Box bbox;

 private:
  bool c0_line(const C0Line& l, V3 p, double cutoff, ExactStats* st, double* d, V3* q, V3* n) const;
  BoxTree tree_;
  bool face(size_t fi, V3 p, double cutoff, ExactStats* st, double* d, V3* q, V3* n) const;
  V3 normal_at(size_t fi, V3 x) const;
};

// partcache.rs:962-970 packed; the 729 values as i16 (nodes x fastest)
int packed_kind(const int16_t* q);  // 0 words, 1 air, 2 solid
void pack_words(const int16_t* q, uint32_t* words);

}  // namespace oracle
