// Oracle trim loops (f64), restating crates/icam-core/src/trim2.rs for rational
// cubic pieces. TEST INFRASTRUCTURE ONLY.
#include "trim.hpp"

#include <algorithm>
#include <cmath>

namespace oracle {

static const int TREE_DEPTH = 10;                 // trim2.rs:99
static const double REF[2] = {0.5137, 0.4871};    // trim2.rs:102

static void bern3(double t, double b[4]) {
  double s = 1.0 - t;
  b[0] = s * s * s;
  b[1] = 3.0 * s * s * t;
  b[2] = 3.0 * s * t * t;
  b[3] = t * t * t;
}

// The rational coordinate k of a piece at t (b_eval of trim2.rs on a rational piece).
double tp_eval(const TPiece& p, int k, double t) {
  // trim2.rs:135-139 b_eval: a constant is itself
  double e0 = p.c[0][k] / p.c[0][2];
  if (e0 == p.c[1][k] / p.c[1][2] && e0 == p.c[2][k] / p.c[2][2] && e0 == p.c[3][k] / p.c[3][2]) return e0;
  double b[4];
  bern3(t, b);
  double n = 0, w = 0;
  for (int i = 0; i < 4; i++) {
    n += b[i] * p.c[i][k];
    w += b[i] * p.c[i][2];
  }
  return n / w;
}

P2 tp_at(const TPiece& p, double t) { return {tp_eval(p, 0, t), tp_eval(p, 1, t)}; }

static double end_val(const TPiece& p, int i, int k) { return p.c[i][k] / p.c[i][2]; }

// The numerator of d(coordinate k)/dt up to a positive factor: N'W - NW' (its sign).
static double tp_dsign(const TPiece& p, int k, double t) {
  double b[4], d[3];
  bern3(t, b);
  double s = 1.0 - t;
  d[0] = s * s;
  d[1] = 2.0 * s * t;
  d[2] = t * t;
  double n = 0, w = 0, n1 = 0, w1 = 0;
  for (int i = 0; i < 4; i++) {
    n += b[i] * p.c[i][k];
    w += b[i] * p.c[i][2];
  }
  for (int i = 0; i < 3; i++) {
    n1 += 3.0 * d[i] * (p.c[i + 1][k] - p.c[i][k]);
    w1 += 3.0 * d[i] * (p.c[i + 1][2] - p.c[i][2]);
  }
  return n1 * w - n * w1;
}

// trim2.rs:1155-1190 crossing: the parameter where coordinate k equals x, when x lies
// in the half-open range [min, max) of its end values. For a rational piece the
// coordinate equals x where the cubic sum_i B_i w_i (c_i - x) vanishes, solved by the
// same safeguarded Newton.
bool tp_crossing(const TPiece& p, int k, double x, double* tout) {
  double p0 = end_val(p, 0, k), p1 = end_val(p, 3, k);
  if (!(std::min(p0, p1) <= x && x < std::max(p0, p1))) return false;
  double a[4];
  for (int i = 0; i < 4; i++) a[i] = p.c[i][k] - x * p.c[i][2];
  auto f = [&](double t) {
    double b[4];
    bern3(t, b);
    return b[0] * a[0] + b[1] * a[1] + b[2] * a[2] + b[3] * a[3];
  };
  auto df = [&](double t) {
    double s = 1.0 - t;
    return 3.0 * (s * s * (a[1] - a[0]) + 2.0 * s * t * (a[2] - a[1]) + t * t * (a[3] - a[2]));
  };
  double lo = 0.0, hi = 1.0;
  double flo = f(0.0);
  if (flo == 0.0) {
    *tout = 0.0;
    return true;
  }
  double t = std::min(std::max((x - p0) / (p1 - p0), 0.0), 1.0);
  for (int it = 0; it < 60; it++) {
    double ft = f(t);
    if (ft == 0.0) {
      *tout = t;
      return true;
    }
    if ((ft < 0.0) == (flo < 0.0)) {
      lo = t;
      flo = ft;
    } else {
      hi = t;
    }
    double d = df(t);
    double nt = d != 0.0 ? t - ft / d : 0.5 * (lo + hi);
    if (!(nt > lo && nt < hi)) nt = 0.5 * (lo + hi);
    if (std::fabs(nt - t) <= 1e-16) {
      *tout = nt;
      return true;
    }
    t = nt;
  }
  *tout = t;
  return true;
}

static std::pair<P2, P2> tp_bbox(const TPiece& p) {
  P2 lo = {INFINITY, INFINITY}, hi = {-INFINITY, -INFINITY};
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 2; k++) {
      double v = end_val(p, i, k);
      lo[k] = std::min(lo[k], v);
      hi[k] = std::max(hi[k], v);
    }
  return {lo, hi};
}

static bool overlaps(P2 alo, P2 ahi, P2 blo, P2 bhi) {
  for (int k = 0; k < 2; k++)
    if (!(alo[k] <= bhi[k] && blo[k] <= ahi[k])) return false;
  return true;
}

// trim2.rs:1141-1150 param_at
static double param_at(const TPiece& p, int k, double x) {
  double a0 = end_val(p, 0, k), a3 = end_val(p, 3, k);
  if (x == a0) return 0.0;
  if (x == a3) return 1.0;
  double t;
  if (tp_crossing(p, k, x, &t)) return t;
  return std::fabs(x - a0) < std::fabs(x - a3) ? 0.0 : 1.0;
}

// trim2.rs:1119-1135 meets_box
static bool meets_box(const TPiece& c, P2 lo, P2 hi) {
  auto bb = tp_bbox(c);
  if (!overlaps(bb.first, bb.second, lo, hi)) return false;
  double u0 = end_val(c, 0, 0), u3 = end_val(c, 3, 0);
  double ta, tb;
  if (u0 == u3) {
    ta = 0.0;
    tb = 1.0;
  } else {
    double a = std::max(lo[0], std::min(u0, u3)), b = std::min(hi[0], std::max(u0, u3));
    ta = param_at(c, 0, a);
    tb = param_at(c, 0, b);
  }
  double va = tp_eval(c, 1, ta), vb = tp_eval(c, 1, tb);
  return std::min(va, vb) <= hi[1] && std::max(va, vb) >= lo[1];
}

// De Casteljau split of a rational cubic piece (homogeneous).
static std::pair<TPiece, TPiece> tp_split(const TPiece& p, double s) {
  std::array<std::array<double, 3>, 4> b = p.c;
  TPiece l, r;
  l.c[0] = b[0];
  r.c[3] = b[3];
  for (int level = 1; level <= 3; level++) {
    for (int i = 0; i <= 3 - level; i++)
      for (int k = 0; k < 3; k++) b[i][k] = (1.0 - s) * b[i][k] + s * b[i + 1][k];
    l.c[level] = b[0];
    r.c[3 - level] = b[3 - level];
  }
  return {l, r};
}

// Pieces are split until each is monotone in both parameters (trim2.rs:22-24): at the
// interior zeros of each coordinate's derivative, found by sign changes on a fine
// grid and bisection.
static void split_monotone(const TPiece& p, std::vector<TPiece>& out) {
  std::vector<double> cuts;
  for (int k = 0; k < 2; k++) {
    const int N = 256;
    double prev = tp_dsign(p, k, 0.0);
    double scale = 0.0;
    for (int i = 0; i <= N; i++) scale = std::max(scale, std::fabs(tp_dsign(p, k, double(i) / N)));
    if (!(scale > 0.0)) continue;
    for (int i = 1; i <= N; i++) {
      double t = double(i) / N;
      double cur = tp_dsign(p, k, t);
      if (std::fabs(cur) <= 1e-13 * scale && i < N) {
        // a root on the grid itself
        double tt = t;
        if (tt > 1e-9 && tt < 1 - 1e-9) cuts.push_back(tt);
        prev = tp_dsign(p, k, t + 0.5 / N);
        continue;
      }
      if ((prev < 0.0 && cur > 0.0) || (prev > 0.0 && cur < 0.0)) {
        double a = double(i - 1) / N, b = t, fa = prev;
        for (int it = 0; it < 100; it++) {
          double m = 0.5 * (a + b);
          double fm = tp_dsign(p, k, m);
          if ((fm < 0.0) == (fa < 0.0)) {
            a = m;
            fa = fm;
          } else {
            b = m;
          }
        }
        double tt = 0.5 * (a + b);
        if (tt > 1e-9 && tt < 1 - 1e-9) cuts.push_back(tt);
      }
      prev = cur;
    }
  }
  std::sort(cuts.begin(), cuts.end());
  TPiece rest = p;
  double done = 0.0;
  for (double t : cuts) {
    if (t - done < 1e-9) continue;
    double s = (t - done) / (1.0 - done);
    auto lr = tp_split(rest, s);
    out.push_back(lr.first);
    rest = lr.second;
    done = t;
  }
  out.push_back(rest);
}

TPiece Trim2::shifted(uint32_t inst) const {
  TPiece c = pieces_[instances_[inst].first];
  P2 s = instances_[inst].second;
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 2; k++) c.c[i][k] += s[k] * c.c[i][2];
  return c;
}

// trim2.rs:1192-1259 parity, with its fixed symbolic perturbation of the path.
bool Trim2::parity(P2 a, P2 b, const std::vector<uint32_t>& among) const {
  uint32_t n = 0;
  bool up = a[1] < b[1];
  bool right = a[0] < b[0];
  for (uint32_t i : among) {
    TPiece c = shifted(i);
    double t;
    if (a[1] != b[1]) {
      if (tp_crossing(c, 0, a[0], &t)) {
        double y = tp_eval(c, 1, t);
        if (up ? (y > a[1] && y <= b[1]) : (y > b[1] && y <= a[1])) n++;
      }
    }
    if (a[0] != b[0]) {
      if (tp_crossing(c, 1, b[1], &t)) {
        double x = tp_eval(c, 0, t);
        auto slope_pos = [&]() {
          double du = tp_dsign(c, 0, t);
          double dv = tp_dsign(c, 1, t);
          if (dv == 0.0) dv = end_val(c, 3, 1) - end_val(c, 0, 1);
          return du * dv > 0.0;
        };
        bool counted;
        if (x == b[0])
          counted = (!slope_pos()) == right;
        else if (x == a[0])
          counted = slope_pos() == right;
        else if (right)
          counted = x > a[0] && x < b[0];
        else
          counted = x > b[0] && x < a[0];
        if (counted) n++;
      }
    }
  }
  return n % 2 == 1;
}

// trim2.rs:1260-1319 place, with the pieces first split monotone.
bool Trim2::build(const std::vector<TPiece>& raw, P2 lo, P2 hi, P2 period, bool inside_left, std::string* err) {
  pieces_.clear();
  for (auto& p : raw) split_monotone(p, pieces_);
  lo_ = lo;
  hi_ = hi;
  period_[0] = period[0];
  period_[1] = period[1];
  inside_left_ = inside_left;
  P2 rlo = lo_, rhi = hi_;
  for (int k = 0; k < 2; k++)
    if (period_[k] > 0) {
      rlo[k] -= period_[k];
      rhi[k] += period_[k];
    }
  instances_.clear();
  for (uint32_t i = 0; i < pieces_.size(); i++) {
    auto bb = tp_bbox(pieces_[i]);
    long ku0 = 0, ku1 = 0, kv0 = 0, kv1 = 0;
    if (period_[0] > 0) {
      ku0 = long(std::ceil((rlo[0] - bb.second[0]) / period_[0]));
      ku1 = long(std::floor((rhi[0] - bb.first[0]) / period_[0]));
    }
    if (period_[1] > 0) {
      kv0 = long(std::ceil((rlo[1] - bb.second[1]) / period_[1]));
      kv1 = long(std::floor((rhi[1] - bb.first[1]) / period_[1]));
    }
    for (long a = ku0; a <= ku1; a++)
      for (long c = kv0; c <= kv1; c++) instances_.push_back({i, P2{a * period_[0], c * period_[1]}});
  }
  std::vector<std::pair<P2, P2>> boxes;
  for (uint32_t i = 0; i < instances_.size(); i++) boxes.push_back(tp_bbox(shifted(i)));
  std::vector<uint32_t> all;
  for (uint32_t i = 0; i < instances_.size(); i++) all.push_back(i);
  P2 root_r = {lo_[0] + (hi_[0] - lo_[0]) * REF[0], lo_[1] + (hi_[1] - lo_[1]) * REF[1]};
  bool root_inside = true;
  if (!pieces_.empty()) {
    // trim2.rs:1331-1346 offset_reference: pieces longest first, each side
    std::vector<const TPiece*> order;
    for (auto& p : pieces_) order.push_back(&p);
    auto chord = [](const TPiece* p) {
      double du = end_val(*p, 3, 0) - end_val(*p, 0, 0), dv = end_val(*p, 3, 1) - end_val(*p, 0, 1);
      return std::sqrt(du * du + dv * dv);
    };
    std::stable_sort(order.begin(), order.end(), [&](const TPiece* a, const TPiece* b) { return chord(a) > chord(b); });
    bool found = false;
    P2 r{};
    bool left = true;
    for (size_t i = 0; i < order.size() && i < 64 && !found; i++)
      for (bool l : {true, false})
        if (!found && offset_from(*order[i], all, l, &r)) {
          found = true;
          left = l;
        }
    if (!found) {
      if (err) *err = "no loop piece gives a settled reference point inside the domain";
      return false;
    }
    root_inside = (left == inside_left_) ^ parity(r, root_r, all);
  }
  cells_.clear();
  Cell root;
  root.lo = lo_;
  root.hi = hi_;
  root.r = root_r;
  root.inside = root_inside;
  root.kind = 0;
  cells_.push_back(root);
  build_cell(0, all, boxes, 0);
  return true;
}

// trim2.rs:1322-1341 build_cell
void Trim2::build_cell(size_t id, const std::vector<uint32_t>& cand, const std::vector<std::pair<P2, P2>>& boxes,
                       int depth) {
  P2 lo = cells_[id].lo, hi = cells_[id].hi, r = cells_[id].r;
  bool inside = cells_[id].inside;
  std::vector<uint32_t> touching;
  for (uint32_t i : cand)
    if (overlaps(lo, hi, boxes[i].first, boxes[i].second)) touching.push_back(i);
  if (touching.empty()) {
    cells_[id].kind = 0;
    return;
  }
  if (depth >= TREE_DEPTH || touching.size() <= 4) {
    cells_[id].kind = 1;
    cells_[id].among = touching;
    return;
  }
  P2 m = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1])};
  std::pair<P2, P2> quads[4] = {{lo, m}, {P2{m[0], lo[1]}, P2{hi[0], m[1]}}, {P2{lo[0], m[1]}, P2{m[0], hi[1]}}, {m, hi}};
  std::array<uint32_t, 4> kids{};
  for (int k = 0; k < 4; k++) {
    P2 qlo = quads[k].first, qhi = quads[k].second;
    P2 qr = {qlo[0] + (qhi[0] - qlo[0]) * REF[0], qlo[1] + (qhi[1] - qlo[1]) * REF[1]};
    bool qin = inside ^ parity(r, qr, touching);
    Cell c;
    c.lo = qlo;
    c.hi = qhi;
    c.r = qr;
    c.inside = qin;
    c.kind = 0;
    size_t kid = cells_.size();
    cells_.push_back(c);
    build_cell(kid, touching, boxes, depth + 1);
    kids[k] = uint32_t(kid);
  }
  cells_[id].kind = 2;
  cells_[id].kids = kids;
}

// trim2.rs:1352-1392 offset_from
bool Trim2::offset_from(const TPiece& p, const std::vector<uint32_t>& all, bool left, P2* out) const {
  double small = std::min(hi_[0] - lo_[0], hi_[1] - lo_[1]);
  auto in_domain = [&](P2 r, double margin) {
    for (int k = 0; k < 2; k++)
      if (!(period_[k] > 0 || (r[k] > lo_[k] + margin && r[k] < hi_[k] - margin))) return false;
    return true;
  };
  P2 m = tp_at(p, 0.5);
  for (int k = 0; k < 2; k++)
    if (period_[k] > 0) {
      double x = std::fmod(m[k] - lo_[k], period_[k]);
      if (x < 0) x += period_[k];
      m[k] = lo_[k] + x;
    }
  P2 a = tp_at(p, 0.49), b = tp_at(p, 0.51);
  double d0 = b[0] - a[0], d1 = b[1] - a[1];
  double l = std::sqrt(d0 * d0 + d1 * d1);
  if (!(l > 0.0)) return false;
  double side = left ? 1.0 : -1.0;
  double n0 = -d1 / l * side, n1 = d0 / l * side;
  double delta = 1e-3 * small;
  while (delta >= 1e-6 * small) {
    P2 r = {m[0] + n0 * delta, m[1] + n1 * delta};
    if (in_domain(r, 0.5 * delta)) {
      double nearest = INFINITY;
      for (uint32_t i : all) nearest = std::min(nearest, dist2_to(i, r));
      if (nearest >= delta * delta * (1.0 - 1e-9)) {
        *out = r;
        return true;
      }
    }
    delta *= 0.5;
  }
  return false;
}

// trim2.rs:1394-1420 dist2_to
double Trim2::dist2_to(uint32_t inst, P2 q) const {
  TPiece c = shifted(inst);
  auto d2 = [&](double t) {
    P2 p = tp_at(c, t);
    return (p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]);
  };
  double best = INFINITY, bt = 0.0;
  for (int k = 0; k <= 16; k++) {
    double t = k / 16.0;
    double d = d2(t);
    if (d < best) {
      best = d;
      bt = t;
    }
  }
  double a = std::max(bt - 1.0 / 16.0, 0.0), b = std::min(bt + 1.0 / 16.0, 1.0);
  for (int it = 0; it < 40; it++) {
    double x = a + 0.381966 * (b - a), y = b - 0.381966 * (b - a);
    if (d2(x) < d2(y))
      b = y;
    else
      a = x;
  }
  return std::min(best, d2(0.5 * (a + b)));
}

// trim2.rs:1433-1457 inside
bool Trim2::inside(double u, double v) const {
  P2 q = {u, v};
  for (int k = 0; k < 2; k++) {
    if (period_[k] > 0) {
      double x = std::fmod(q[k] - lo_[k], period_[k]);
      if (x < 0) x += period_[k];
      q[k] = lo_[k] + x;
    } else {
      q[k] = std::min(std::max(q[k], lo_[k]), hi_[k]);
    }
  }
  if (pieces_.empty()) return true;
  size_t id = 0;
  for (;;) {
    const Cell& c = cells_[id];
    if (c.kind == 0) return c.inside;
    if (c.kind == 1) return c.inside ^ parity(c.r, q, c.among);
    P2 m = {0.5 * (c.lo[0] + c.hi[0]), 0.5 * (c.lo[1] + c.hi[1])};
    int k = int(q[0] >= m[0]) + 2 * int(q[1] >= m[1]);
    id = c.kids[k];
  }
}

// trim2.rs:1570-1612 box_class / class_in
int Trim2::box_class(P2 lo, P2 hi) const {
  if (pieces_.empty()) return 1;
  return class_in(0, lo, hi);
}

int Trim2::class_in(size_t id, P2 lo, P2 hi) const {
  const Cell& c = cells_[id];
  P2 ilo = {std::max(lo[0], c.lo[0]), std::max(lo[1], c.lo[1])};
  P2 ihi = {std::min(hi[0], c.hi[0]), std::min(hi[1], c.hi[1])};
  if (c.kind == 0) return c.inside ? 1 : 0;
  if (c.kind == 1) {
    double g = 1e-12 * (std::fabs(hi_[0] - lo_[0]) + std::fabs(hi_[1] - lo_[1]));
    P2 glo = {ilo[0] - g, ilo[1] - g}, ghi = {ihi[0] + g, ihi[1] + g};
    for (uint32_t i : c.among)
      if (meets_box(shifted(i), glo, ghi)) return -1;
    P2 m = {0.5 * (ilo[0] + ihi[0]), 0.5 * (ilo[1] + ihi[1])};
    return (c.inside ^ parity(c.r, m, c.among)) ? 1 : 0;
  }
  int answer = -2;
  for (uint32_t k : c.kids) {
    const Cell& kc = cells_[k];
    if (!overlaps(kc.lo, kc.hi, lo, hi)) continue;
    int a = class_in(k, lo, hi);
    if (a == -1) return -1;
    if (answer == -2)
      answer = a;
    else if (answer != a)
      return -1;
  }
  return answer == -2 ? -1 : answer;
}

}  // namespace oracle
