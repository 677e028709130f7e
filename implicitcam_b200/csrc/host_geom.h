// Host-side geometry used while packing a solid: vectors, rational Bezier patches and
// curves, interval derivative bounds, and the trim-tree builder. Double precision.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

namespace icam {

struct V {
  double x = 0, y = 0, z = 0;
  V() = default;
  V(double a, double b, double c) : x(a), y(b), z(c) {}
  V operator+(V o) const { return {x + o.x, y + o.y, z + o.z}; }
  V operator-(V o) const { return {x - o.x, y - o.y, z - o.z}; }
  V operator*(double s) const { return {x * s, y * s, z * s}; }
  V operator-() const { return {-x, -y, -z}; }
  double dot(V o) const { return x * o.x + y * o.y + z * o.z; }
  V cross(V o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
  double len() const { return std::sqrt(dot(*this)); }
  V unit() const {
    double l = len();
    return l > 0 ? *this * (1.0 / l) : *this;
  }
  double& operator[](int k) { return k == 0 ? x : (k == 1 ? y : z); }
  double operator[](int k) const { return k == 0 ? x : (k == 1 ? y : z); }
};

using H = std::array<double, 4>;
inline V hv(const H& h) { return {h[0] / h[3], h[1] / h[3], h[2] / h[3]}; }

struct Bx {
  V lo{1e300, 1e300, 1e300}, hi{-1e300, -1e300, -1e300};
  void add(V p) {
    for (int k = 0; k < 3; k++) {
      lo[k] = std::min(lo[k], p[k]);
      hi[k] = std::max(hi[k], p[k]);
    }
  }
  void add(const Bx& b) {
    add(b.lo);
    add(b.hi);
  }
  double dist(V p) const {
    V d(std::max(std::max(lo.x - p.x, p.x - hi.x), 0.0), std::max(std::max(lo.y - p.y, p.y - hi.y), 0.0),
        std::max(std::max(lo.z - p.z, p.z - hi.z), 0.0));
    return d.len();
  }
  V mid() const { return (lo + hi) * 0.5; }
};

// A bicubic rational patch: p[i][j], i along u; its rectangle in the face's parameters.
struct Bicubic {
  H p[4][4];
  double u0 = 0, u1 = 1, v0 = 0, v1 = 1;
  Bx box() const {
    Bx b;
    for (auto& r : p)
      for (auto& h : r) b.add(hv(h));
    return b;
  }
  // point and first/second derivatives at local (s, t)
  void eval(double s, double t, V* P, V* Ps, V* Pt, V* Pss, V* Pst, V* Ptt) const;
  void split_u(double s, Bicubic* l, Bicubic* r) const;
  void split_v(double t, Bicubic* l, Bicubic* r) const;
};

// Raises a Bezier control polygon (homogeneous) by one degree.
std::vector<H> elevate(const std::vector<H>& q);

// Interval derivative bounds and the convexity certificate of a bicubic
// (surface3.rs:814-925 patch_bounds, restated): false when a weight is not positive.
bool patch_bounds(const Bicubic& pa, double* sa, double* sb, double* lam, double d2[3][3][2], double* rho);

// The same for a rational cubic curve piece (surface3.rs:933-965 bez_bounds).
bool piece_bounds(const H c[4], double* lam, double d2[3][2]);

// Rational cubic piece in 3D.
struct Cubic3 {
  H c[4];
  void eval(double s, V* P, V* D1) const;
  void split(double s, Cubic3* l, Cubic3* r) const;
  double turning() const;
  double thickness() const;
  Bx box() const {
    Bx b;
    for (auto& h : c) b.add(hv(h));
    return b;
  }
};

// Whether the piece's convexity certificate (the device's piece_convex) holds for every
// point within `need` of its control-point box.
bool piece_certifies(const Cubic3& z, double need);

// ---------------------------------------------------------------- trim trees

// A loop piece in a face's (u, v): rational cubic, (u w, v w, w).
struct TP {
  double c[4][3];
};

struct TCell {
  double lo[2], hi[2], r[2];
  int inside, kind;  // kind 0 leaf, 1 crossed, 2 split
  std::vector<int> among;
  int kids[4] = {-1, -1, -1, -1};
};

// One face's loops as monotone pieces with periodic copies and a cell tree whose
// cells hold a reference point and its answer (trim2.rs:1105-1341, built here for
// exact rational pieces).
struct TrimTree {
  std::vector<TP> pieces;
  std::vector<std::pair<int, std::array<double, 2>>> inst;
  std::vector<TCell> cells;
  double lo[2], hi[2], period[2];
  bool inside_left = true;
  bool build(const std::vector<TP>& raw, const double lo_[2], const double hi_[2], const double per[2], bool left,
             std::string* err);
  bool inside(double u, double v) const;
  int box_class(const double lo_[2], const double hi_[2]) const;  // 1 in, 0 out, -1 straddles
  TP shifted(int i) const;
  bool parity(const double a[2], const double b[2], const std::vector<int>& among) const;

 private:
  void build_cell(int id, const std::vector<int>& cand, const std::vector<std::array<double, 4>>& boxes, int depth);
  bool offset_point(const TP& p, const std::vector<int>& all, bool left, double out[2]) const;
  double dist2(int inst, const double q[2]) const;
  int class_in(int id, const double lo_[2], const double hi_[2]) const;
};

// Evaluation helpers shared by the builder and its self-check.
double tp_coord(const TP& p, int k, double t);
double tp_dnum(const TP& p, int k, double t);
bool tp_cross(const TP& p, int k, double x, double* t);

}  // namespace icam
