// Oracle exact signed distance (f64). TEST INFRASTRUCTURE ONLY.
#include "exact.hpp"

#include <algorithm>
#include <cmath>
#include <queue>

namespace oracle {

static const double DIST_EPS = 1e-9;   // surface3.rs:975
static const int SEARCH_NEWTON = 12;   // surface3.rs:972
static const double FLAT = 0.35;       // curve3.rs:1015

// surface3.rs:40-48 axial
struct Axial {
  double theta, rho, h;
  V3 er, et;
};
static Axial axial(const Frame& f, V3 p) {
  V3 l = f.local(p);
  double rho = std::sqrt(l.x * l.x + l.y * l.y);
  double theta = rho > 0.0 ? std::atan2(l.y, l.x) : 0.0;
  double s = std::sin(theta), c = std::cos(theta);
  return {theta, rho, l.z, f.dir(V3(c, s, 0.0)), f.dir(V3(-s, c, 0.0))};
}

// ---------------------------------------------------------------- analytic surfaces

// surface3.rs:85-129 Surf::foot
V3 Surf::foot(V3 p) const {
  switch (kind) {
    case PLANE:
      return p - f.z * (p - f.o).dot(f.z);
    case CYLINDER: {
      Axial ax = axial(f, p);
      return f.o + ax.er * a + f.z * ax.h;
    }
    case CONE: {
      Axial ax = axial(f, p);
      double sa = std::sin(b), ca = std::cos(b);
      double ha = -a / std::tan(b);
      double s = ax.rho * sa + (ax.h - ha) * ca;
      if (s <= 0.0) return f.o + f.z * ha;
      return f.o + ax.er * (s * sa) + f.z * (ha + s * ca);
    }
    case SPHERE: {
      V3 d = p - f.o;
      double l = d.len();
      return l > 0.0 ? f.o + d * (a / l) : f.o + f.x * a;
    }
    case TORUS: {
      double major = a, minor = b;
      Axial ax = axial(f, p);
      V3 c = f.o + ax.er * major;
      V3 d = p - c;
      double l = d.len();
      V3 q = l > 0.0 ? c + d * (minor / l) : c + ax.er * minor;
      if ((q - f.o).dot(ax.er) >= 0.0 || std::fabs(major) > minor) return q;
      double h = std::sqrt(std::max(minor * minor - major * major, 0.0));
      return ax.h >= 0.0 ? f.o + f.z * h : f.o - f.z * h;
    }
    default: {
      SurfHit h;
      if (ns->closest(p, INF, &h)) return h.q;
      return p;
    }
  }
}

// surface3.rs:132-148 Surf::normal
V3 Surf::normal(V3 x) const {
  switch (kind) {
    case PLANE:
      return f.z;
    case CYLINDER:
      return axial(f, x).er;
    case CONE: {
      Axial ax = axial(f, x);
      return ax.er * std::cos(b) - f.z * std::sin(b);
    }
    case SPHERE:
      return (x - f.o).unit();
    case TORUS: {
      Axial ax = axial(f, x);
      return (x - (f.o + ax.er * a)).unit();
    }
    default: {
      SurfHit h;
      if (ns->closest(x, INF, &h)) return h.n;
      return V3(0, 0, 1);
    }
  }
}

// The parameters the face's loops are in (Analytic::uv, trim2.rs:1904-1933, with the
// angle itself as the angular parameter).
void Surf::uv(V3 q, double* u, double* v) const {
  Axial ax = axial(f, q);
  switch (kind) {
    case PLANE: {
      V3 l = f.local(q);
      *u = l.x;
      *v = l.y;
      return;
    }
    case CYLINDER:
      *u = ax.theta;
      *v = ax.h;
      return;
    case CONE: {
      double sa = std::sin(b), ca = std::cos(b);
      double ha = -a / std::tan(b);
      double s = std::max(ax.rho * sa + (ax.h - ha) * ca, 0.0);
      *u = ax.theta;
      *v = ha + s * ca;
      return;
    }
    case SPHERE:
      *u = ax.theta;
      *v = std::atan2(ax.h, ax.rho);
      return;
    case TORUS:
      *u = ax.theta;
      *v = std::atan2(ax.h, ax.rho - a);
      return;
    default:
      *u = *v = 0;
  }
}

// ---------------------------------------------------------------- B-spline surfaces

int NurbsSurf::build(int i0, int i1, int j0, int j1) {
  int id = int(nodes.size());
  nodes.push_back({});
  nodes[id].i0 = i0;
  nodes[id].i1 = i1;
  nodes[id].j0 = j0;
  nodes[id].j1 = j1;
  if (i1 - i0 == 1 && j1 - j0 == 1) {
    nodes[id].box = span(i0, j0).bbox();
    return id;
  }
  int im = (i0 + i1) / 2, jm = (j0 + j1) / 2;
  std::vector<std::pair<int, int>> ir, jr;
  if (i1 - i0 > 1)
    ir = {{i0, im}, {im, i1}};
  else
    ir = {{i0, i1}};
  if (j1 - j0 > 1)
    jr = {{j0, jm}, {jm, j1}};
  else
    jr = {{j0, j1}};
  std::vector<int> kids;
  for (auto& a : ir)
    for (auto& c : jr) kids.push_back(build(a.first, a.second, c.first, c.second));
  Box b = empty_box();
  for (int k : kids) {
    b.first = vmin(b.first, nodes[k].box.first);
    b.second = vmax(b.second, nodes[k].box.second);
  }
  nodes[id].box = b;
  nodes[id].kids = kids;
  return id;
}

void NurbsSurf::build_tree() {
  nodes.clear();
  build(0, nsu, 0, nsv);
}

// surface3.rs:587-591 Creases::touches
bool NurbsSurf::touches(const Patch& pa) const {
  auto on = [](double x, const std::vector<double>& lines, double a, double b) {
    for (double c : lines)
      if (std::fabs(x - c) <= 1e-12 * std::max(std::fabs(b - a), std::fabs(c))) return true;
    return false;
  };
  return on(pa.u0, cu, pa.u0, pa.u1) || on(pa.u1, cu, pa.u0, pa.u1) || on(pa.v0, cv, pa.v0, pa.v1) ||
         on(pa.v1, cv, pa.v0, pa.v1);
}

// surface3.rs:1168-1173 span_of
int NurbsSurf::span_of(const std::vector<double>& br, double x) const {
  int n = int(br.size()) - 1;
  for (int i = n - 1; i >= 0; i--)
    if (br[i] <= x) return i;
  return 0;
}

// surface3.rs:1175-1181 eval at global parameters
SEval NurbsSurf::eval(double u, double v) const {
  int a = span_of(ub, u), b = span_of(vb, v);
  const Patch& pa = span(a, b);
  double s = (u - pa.u0) / (pa.u1 - pa.u0), t = (v - pa.v0) / (pa.v1 - pa.v0);
  SEval e = pa.eval(std::min(std::max(s, 0.0), 1.0), std::min(std::max(t, 0.0), 1.0));
  double x = 1.0 / (pa.u1 - pa.u0), y = 1.0 / (pa.v1 - pa.v0);
  return {e.p, e.ps * x, e.pt * y, e.pss * (x * x), e.pst * (x * y), e.ptt * (y * y)};
}

namespace {
// surface3.rs:1206-1212 PatchItem (min-heap on lb)
struct Item {
  double lb;
  int node;  // >= 0: a quadtree node; -1: the patch
  Patch pa;
  int depth;
  bool inside;
};
struct ItemCmp {
  bool operator()(const Item* a, const Item* b) const { return a->lb > b->lb; }
};
}  // namespace

// surface3.rs:1214-1297 closest_trimmed
bool NurbsSurf::closest_trimmed(V3 p, double cutoff, const Trim2* trim, SurfHit* hit, bool* complete,
                                int* pops_out) const {
  bool have = false;
  SurfHit best{};
  double best_d = cutoff;
  std::vector<std::unique_ptr<Item>> store;
  std::priority_queue<Item*, std::vector<Item*>, ItemCmp> heap;
  auto push = [&](double lb, int node, const Patch* pa, int depth, bool inside) {
    store.emplace_back(new Item{lb, node, pa ? *pa : Patch(), depth, inside});
    heap.push(store.back().get());
  };
  push(box_dist(p, bbox()), 0, nullptr, 0, false);
  int pops = 0;
  auto answer = [&](const SurfHit& h) {
    if (!have || h.dist < best.dist) {
      best = h;
      have = true;
    }
  };
  auto klass = [&](double u0, double v0, double u1, double v1) { return trim->box_class({u0, v0}, {u1, v1}); };
  *complete = true;
  while (!heap.empty()) {
    Item* it = heap.top();
    heap.pop();
    double lb = it->lb;
    if (lb >= best_d - DIST_EPS || best_d <= DIST_EPS) break;
    pops++;
    if (pops > 20000) {
      *complete = false;
      break;
    }
    if (it->node >= 0) {
      const QNode& n = nodes[it->node];
      int state = it->inside ? 1 : klass(ub[n.i0], vb[n.j0], ub[n.i1], vb[n.j1]);
      if (state == 0) continue;
      bool now_in = state == 1;
      if (n.kids.empty()) {
        const Patch& pa = span(n.i0, n.j0);
        double lbp = std::max(box_dist(p, pa.bbox()), lb);
        if (lbp < best_d - DIST_EPS) push(lbp, -1, &pa, 0, now_in);
      } else {
        for (int k : n.kids) {
          double lbk = box_dist(p, nodes[k].box);
          if (lbk < best_d - DIST_EPS) push(lbk, k, nullptr, 0, now_in);
        }
      }
      continue;
    }
    const Patch& pa = it->pa;
    int state = it->inside ? 1 : klass(pa.u0, pa.v0, pa.u1, pa.v1);
    if (state == 0) continue;
    bool now_in = state == 1;
    auto st = pa.newton_capped(p, 0.5, 0.5, SEARCH_NEWTON);
    SEval e = pa.eval(st.first, st.second);
    double d = (e.p - p).len();
    V3 n = e.ps.cross(e.pt).unit();
    double u = pa.u0 + st.first * (pa.u1 - pa.u0), v = pa.v0 + st.second * (pa.v1 - pa.v0);
    if (d < best_d && (now_in || trim->inside(u, v))) {
      best_d = d;
      if (critical(p, e)) {
        answer({e.p, d, u, v, n});
      } else {
        SurfHit h;
        if (descend(p, u, v, false, &h)) {
          if (h.dist <= d && trim->inside(h.u, h.v)) {
            best_d = std::min(best_d, h.dist);
            answer(h);
          }
        }
      }
    }
    double slab = slab_bound(pa, p, d > 1e-12 ? (p - e.p) * (1.0 / d) : n);
    if (slab >= best_d - DIST_EPS || it->depth >= 40) continue;
    // a patch touching a collapsed side is never cleared: the distance's minimum at a
    // pole need not be a critical point of the patch's parameters
    if (!touches(pa) && pa.no_critical_point(p)) continue;
    Patch q[4];
    pa.quarters(q);
    for (int k = 0; k < 4; k++) {
      double lbq = std::max(box_dist(p, q[k].bbox()), slab);
      if (lbq < best_d - DIST_EPS) push(lbq, -1, &q[k], it->depth + 1, now_in);
    }
  }
  *pops_out = pops;
  if (have) *hit = best;
  return have;
}

// surface3.rs:1314-1366 descend
bool NurbsSurf::descend(V3 p, double u, double v, bool border, SurfHit* hit) const {
  int a = span_of(ub, u), b = span_of(vb, v);
  const Patch* pa = &span(a, b);
  double s = (u - pa->u0) / (pa->u1 - pa->u0), t = (v - pa->v0) / (pa->v1 - pa->v0);
  for (int it = 0; it < 16; it++) {
    auto st = pa->newton_capped(p, std::min(std::max(s, 0.0), 1.0), std::min(std::max(t, 0.0), 1.0), 40);
    double ns = st.first, nt = st.second;
    SEval e = pa->eval(ns, nt);
    if (critical(p, e)) {
      *hit = {e.p, (e.p - p).len(), pa->u0 + ns * (pa->u1 - pa->u0), pa->v0 + nt * (pa->v1 - pa->v0),
              e.ps.cross(e.pt).unit()};
      return true;
    }
    V3 r = e.p - p;
    double gs = r.dot(e.ps), gt = r.dot(e.pt);
    bool moved = false;
    int na = a, nb = b;
    if (ns >= 1.0 && gs < 0.0 && a + 1 < nsu) {
      na = a + 1;
      s = 0.0;
      moved = true;
    } else if (ns <= 0.0 && gs > 0.0 && a > 0) {
      na = a - 1;
      s = 1.0;
      moved = true;
    } else {
      s = ns;
    }
    if (nt >= 1.0 && gt < 0.0 && b + 1 < nsv) {
      nb = b + 1;
      t = 0.0;
      moved = true;
    } else if (nt <= 0.0 && gt > 0.0 && b > 0) {
      nb = b - 1;
      t = 1.0;
      moved = true;
    } else {
      t = nt;
    }
    if (!moved) {
      if (border) {
        *hit = {e.p, r.len(), pa->u0 + ns * (pa->u1 - pa->u0), pa->v0 + nt * (pa->v1 - pa->v0),
                e.ps.cross(e.pt).unit()};
        return true;
      }
      return false;
    }
    a = na;
    b = nb;
    pa = &span(a, b);
  }
  return false;
}

// surface3.rs:1444-1499 closest (untrimmed)
bool NurbsSurf::closest(V3 p, double cutoff, SurfHit* hit) const {
  bool have = false;
  SurfHit best{};
  double best_d = cutoff;
  std::vector<std::unique_ptr<Item>> store;
  std::priority_queue<Item*, std::vector<Item*>, ItemCmp> heap;
  auto push = [&](double lb, int node, const Patch* pa, int depth) {
    store.emplace_back(new Item{lb, node, pa ? *pa : Patch(), depth, false});
    heap.push(store.back().get());
  };
  push(box_dist(p, bbox()), 0, nullptr, 0);
  int pops = 0;
  while (!heap.empty()) {
    Item* it = heap.top();
    heap.pop();
    double lb = it->lb;
    if (lb >= best_d - DIST_EPS || best_d <= DIST_EPS) break;
    if (++pops > 20000) break;
    if (it->node >= 0) {
      const QNode& n = nodes[it->node];
      if (n.kids.empty()) {
        const Patch& pa = span(n.i0, n.j0);
        double lbp = std::max(box_dist(p, pa.bbox()), lb);
        if (lbp < best_d - DIST_EPS) push(lbp, -1, &pa, 0);
      } else {
        for (int k : n.kids) {
          double lbk = box_dist(p, nodes[k].box);
          if (lbk < best_d - DIST_EPS) push(lbk, k, nullptr, 0);
        }
      }
      continue;
    }
    const Patch& pa = it->pa;
    auto st = pa.newton_capped(p, 0.5, 0.5, SEARCH_NEWTON);
    SEval e = pa.eval(st.first, st.second);
    double d = (e.p - p).len();
    V3 n = e.ps.cross(e.pt).unit();
    if (d < best_d) {
      best_d = d;
      best = {e.p, d, pa.u0 + st.first * (pa.u1 - pa.u0), pa.v0 + st.second * (pa.v1 - pa.v0), n};
      have = true;
    }
    double slab = slab_bound(pa, p, d > 1e-12 ? (p - e.p) * (1.0 / d) : n);
    if (slab >= best_d - DIST_EPS || it->depth >= 40) continue;
    Patch q[4];
    pa.quarters(q);
    for (int k = 0; k < 4; k++) {
      double lbq = std::max(box_dist(p, q[k].bbox()), slab);
      if (lbq < best_d - DIST_EPS) push(lbq, -1, &q[k], it->depth + 1);
    }
  }
  if (have) *hit = best;
  return have;
}

// ---------------------------------------------------------------- edges

// curve3.rs:408-471 Spline3::closest (branch and bound over the flat pieces)
bool Spline3::closest(V3 p, double cutoff, Foot3* out) const {
  bool have = false;
  Foot3 best{};
  double best_d = cutoff;
  struct E {
    double lb;
    size_t i;
    Bez3 z;
    int depth;
  };
  std::vector<E> stack;
  for (size_t i = 0; i < pieces.size(); i++) {
    const Bez3& z = pieces[i];
    double lb = std::max(box_dist(p, boxes[i]), seg_dist3(p, z.start(), z.end()) - thick[i]);
    if (lb < best_d) stack.push_back({lb, i, z, 0});
  }
  auto srt = [&]() { std::stable_sort(stack.begin(), stack.end(), [](const E& a, const E& b) { return a.lb > b.lb; }); };
  srt();
  int popped = 0;
  while (!stack.empty()) {
    E en = stack.back();
    stack.pop_back();
    if (en.lb >= best_d - 1e-12) continue;
    if (++popped > 4096) break;
    const Bez3& z = en.z;
    V3 a = z.start(), b = z.end(), ab = b - a;
    double l2 = ab.dot(ab);
    double f = l2 > 0.0 ? std::min(std::max((p - a).dot(ab) / l2, 0.0), 1.0) : 0.5;
    for (double s0 : {f, 0.0, 1.0, -1.0, 2.0}) {
      double s = s0 < 0.0 ? 0.0 : (s0 > 1.0 ? 1.0 : z.newton(p, s0));
      Eval3 e = z.eval(s);
      double d = (p - e.p).len();
      if (d < best_d) {
        best_d = d;
        bool last = en.i == pieces.size() - 1 && s >= 1.0 && z.t1 == pieces[en.i].t1;
        bool first = en.i == 0 && s <= 0.0 && z.t0 == pieces[en.i].t0;
        int near = first ? START : (last ? END : INTERIOR);
        best = {e.p, d, z.t0 + s * (z.t1 - z.t0), near, e.d1.unit()};
        have = true;
      }
    }
    if (en.depth < 40 && z.thickness() > 1e-12) {
      auto lr = z.split(0.5);
      for (const Bez3* c : {&lr.first, &lr.second}) {
        double lbc = seg_dist3(p, c->start(), c->end()) - c->thickness();
        if (lbc < best_d - 1e-12) stack.push_back({lbc, en.i, *c, en.depth + 1});
      }
      srt();
    }
  }
  if (have) *out = best;
  return have;
}

// curve3.rs:580-585 swept
static double swept(double t0, double t, double sweep) {
  double d = sweep >= 0.0 ? t - t0 : t0 - t;
  double m = std::fmod(d, 2.0 * PI);
  if (m < 0) m += 2.0 * PI;
  return m;
}

// curve3.rs:502-521 Edge3::at
V3 Edge3::at(double s) const {
  if (kind == 0) return a + (b - a) * s;
  if (kind == 1) {
    double t = t0 + s * sweep;
    return f.world(V3(r * std::cos(t), r * std::sin(t), 0.0));
  }
  double n = double(sp->pieces.size());
  size_t k = std::min(size_t(s * n), sp->pieces.size() - 1);
  return sp->pieces[k].eval(s * n - double(k)).p;
}

// curve3.rs:658-675 tangent_at
V3 Edge3::tangent_at(double s) const {
  if (kind == 0) return (b - a).unit();
  if (kind == 1) {
    double t = t0 + s * sweep;
    return f.dir(V3(-std::sin(t), std::cos(t), 0.0)) * (sweep >= 0 ? 1.0 : -1.0);
  }
  double n = double(sp->pieces.size());
  size_t k = std::min(size_t(s * n), sp->pieces.size() - 1);
  return sp->pieces[k].eval(s * n - double(k)).d1.unit();
}

// curve3.rs:525-598 Edge3::closest (lines, arcs, splines)
Foot3 Edge3::closest(V3 p) const {
  if (kind == 0) {
    V3 ab = b - a;
    double l2 = ab.dot(ab);
    double t = l2 > 0.0 ? std::min(std::max((p - a).dot(ab) / l2, 0.0), 1.0) : 0.0;
    V3 q = a + ab * t;
    int near = t <= 0.0 ? START : (t >= 1.0 ? END : INTERIOR);
    return {q, (p - q).len(), t, near, ab.unit()};
  }
  if (kind == 1) {
    V3 l = f.local(p);
    bool full = std::fabs(std::fabs(sweep) - 2.0 * PI) < 1e-12;
    double t = std::atan2(l.y, l.x);
    double sg = sweep >= 0 ? 1.0 : -1.0;
    auto tan = [&](double tt) { return f.dir(V3(-std::sin(tt), std::cos(tt), 0.0)) * sg; };
    if ((l.x != 0.0 || l.y != 0.0) && (full || swept(t0, t, sweep) <= std::fabs(sweep))) {
      V3 q = f.world(V3(r * std::cos(t), r * std::sin(t), 0.0));
      return {q, (p - q).len(), t, INTERIOR, tan(t)};
    }
    V3 qa = at(0.0), qb = at(1.0);
    if ((p - qa).len() <= (p - qb).len()) return {qa, (p - qa).len(), t0, START, tan(t0)};
    return {qb, (p - qb).len(), t0 + sweep, END, tan(t0 + sweep)};
  }
  Foot3 o{};
  sp->closest(p, INF, &o);
  return o;
}

// curve3.rs:600-607 closest_below
bool Edge3::closest_below(V3 p, double cutoff, Foot3* out) const {
  if (kind == 2) return sp->closest(p, cutoff, out);
  Foot3 f0 = closest(p);
  if (!(f0.dist < cutoff)) return false;
  *out = f0;
  return true;
}

// curve3.rs:677-712 Edge3::bbox
Box Edge3::bbox() const {
  Box bx = empty_box();
  if (kind == 0) {
    grow(bx, a);
    grow(bx, b);
  } else if (kind == 1) {
    V3 axes[3] = {V3(1, 0, 0), V3(0, 1, 0), V3(0, 0, 1)};
    for (V3 ax : axes) {
      double e = std::sqrt(std::max(1.0 - std::pow(f.z.dot(ax), 2), 0.0)) * r;
      grow(bx, f.o + ax * e);
      grow(bx, f.o - ax * e);
    }
  } else {
    for (auto& b2 : sp->boxes) {
      grow(bx, b2.first);
      grow(bx, b2.second);
    }
  }
  return bx;
}

// ---------------------------------------------------------------- box tree

// solid3.rs:108-140 BoxTree::new / build
void BoxTree::init(const std::vector<Box>& boxes) {
  ids_.resize(boxes.size());
  for (size_t i = 0; i < boxes.size(); i++) ids_[i] = i;
  std::stable_sort(ids_.begin(), ids_.end(), [&](size_t a, size_t b) {
    return (boxes[a].first.x + boxes[a].second.x) < (boxes[b].first.x + boxes[b].second.x);
  });
  boxes_.clear();
  for (size_t i : ids_) boxes_.push_back(boxes[i]);
  at_.assign(ids_.size(), 0);
  for (size_t k = 0; k < ids_.size(); k++) at_[ids_[k]] = k;
  nodes_.clear();
  if (!boxes_.empty()) build(0, 0, boxes_.size());
}

Box BoxTree::build(size_t k, size_t a, size_t b) {
  if (nodes_.size() <= k) nodes_.resize(k + 1);
  Box bx;
  if (b - a <= 4) {
    bx = {V3(1.79e308, 1.79e308, 1.79e308), V3(-1.79e308, -1.79e308, -1.79e308)};
    for (size_t i = a; i < b; i++) {
      bx.first = vmin(bx.first, boxes_[i].first);
      bx.second = vmax(bx.second, boxes_[i].second);
    }
  } else {
    size_t m = (a + b) / 2;
    Box l = build(2 * k + 1, a, m), r = build(2 * k + 2, m, b);
    bx = {vmin(l.first, r.first), vmax(l.second, r.second)};
  }
  nodes_[k] = {bx, a, b};
  return bx;
}

// solid3.rs:167-198 nearest_first
template <class F>
void BoxTree::nearest_first(V3 p, double bound, F&& f) const {
  if (nodes_.empty()) return;
  struct N {
    double lb;
    size_t k;
    bool leaf;
  };
  auto cmp = [](const N& a, const N& b) { return a.lb > b.lb; };
  std::priority_queue<N, std::vector<N>, decltype(cmp)> heap(cmp);
  heap.push({box_dist(p, nodes_[0].b), 0, false});
  while (!heap.empty()) {
    N n = heap.top();
    heap.pop();
    if (n.lb >= bound) break;
    if (n.leaf) {
      bound = f(ids_[n.k]);
      continue;
    }
    const Node& nd = nodes_[n.k];
    if (nd.e - nd.a <= 4) {
      for (size_t i = nd.a; i < nd.e; i++) {
        double d = box_dist(p, boxes_[i]);
        if (d < bound) heap.push({d, i, true});
      }
    } else {
      for (size_t c : {2 * n.k + 1, 2 * n.k + 2}) {
        double d = box_dist(p, nodes_[c].b);
        if (d < bound) heap.push({d, c, false});
      }
    }
  }
}

// ---------------------------------------------------------------- the solid

static Frame frame_of(const IcamFrame& f) {
  return {V3(f.o[0], f.o[1], f.o[2]), V3(f.z[0], f.z[1], f.z[2]), V3(f.x[0], f.x[1], f.x[2])};
}

// solid3.rs:1211-1278 face_box
static Box face_box(const Face& f, const std::vector<EdgeRec>& edges) {
  Box bx = empty_box();
  V3 axes[3] = {V3(1, 0, 0), V3(0, 1, 0), V3(0, 0, 1)};
  auto circle_box = [&](V3 c, V3 z, double r) {
    for (V3 ax : axes) {
      double e = std::sqrt(std::max(1.0 - std::pow(z.dot(ax), 2), 0.0)) * r;
      grow(bx, c + ax * e);
      grow(bx, c - ax * e);
    }
  };
  const Surf& s = f.surf;
  switch (s.kind) {
    case PLANE:
      for (auto& lp : f.loops)
        for (auto& u : lp) {
          grow(bx, edges[u.first].box.first);
          grow(bx, edges[u.first].box.second);
        }
      break;
    case CYLINDER:
    case CONE: {
      double h0 = 1.79e308, h1 = -1.79e308;
      for (auto& lp : f.loops)
        for (auto& u : lp) {
          V3 a = edges[u.first].box.first, b = edges[u.first].box.second;
          for (int k = 0; k < 8; k++) {
            V3 q((k & 1) ? b.x : a.x, (k & 2) ? b.y : a.y, (k & 4) ? b.z : a.z);
            double h = (q - s.f.o).dot(s.f.z);
            h0 = std::min(h0, h);
            h1 = std::max(h1, h);
          }
        }
      for (double h : {h0, h1}) {
        double rad = s.kind == CONE ? std::fabs(s.a + h * std::tan(s.b)) : s.a;
        circle_box(s.f.o + s.f.z * h, s.f.z, rad);
      }
      break;
    }
    case SPHERE:
      grow(bx, s.f.o - V3(s.a, s.a, s.a));
      grow(bx, s.f.o + V3(s.a, s.a, s.a));
      break;
    case TORUS:
      for (double h : {-s.b, s.b}) circle_box(s.f.o + s.f.z * h, s.f.z, s.a + s.b);
      break;
    default: {
      Box b = s.ns->bbox();
      grow(bx, b.first);
      grow(bx, b.second);
    }
  }
  return bx;
}

bool Exact::init(const IcamSolidDesc* d, std::string* err) {
  tol = d->tol;
  faces.clear();
  edges.clear();
  verts.clear();
  for (int i = 0; i < d->n_verts; i++) verts.push_back({V3(d->verts[3 * i], d->verts[3 * i + 1], d->verts[3 * i + 2]), V3()});
  for (int i = 0; i < d->n_edges; i++) {
    const IcamEdgeDesc& e = d->edges[i];
    EdgeRec r;
    r.curve.kind = e.kind;
    r.faces[0] = e.f0;
    r.faces[1] = e.f1;
    r.v[0] = e.v0;
    r.v[1] = e.v1;
    if (e.kind == ICAM_EDGE_LINE) {
      r.curve.a = V3(e.a[0], e.a[1], e.a[2]);
      r.curve.b = V3(e.b[0], e.b[1], e.b[2]);
    } else if (e.kind == ICAM_EDGE_ARC) {
      r.curve.f = frame_of(e.f);
      r.curve.r = e.r;
      r.curve.t0 = e.t0;
      r.curve.sweep = e.sweep;
    } else {
      // curve3.rs:345-372 Spline3::new: the pieces flattened (FLAT) with their boxes
      auto sp = std::make_shared<Spline3>();
      std::vector<Bez3> stack;
      for (int k = e.n_pieces - 1; k >= 0; k--) {
        Bez3 z;
        const double* c = d->cpieces + size_t(e.first_piece + k) * (e.degree + 1) * 4;
        for (int j = 0; j <= e.degree; j++) z.pw.push_back({c[4 * j], c[4 * j + 1], c[4 * j + 2], c[4 * j + 3]});
        z.t0 = k;
        z.t1 = k + 1;
        stack.push_back(z);
      }
      while (!stack.empty()) {
        Bez3 z = stack.back();
        stack.pop_back();
        if (z.turning() <= FLAT || std::fabs(z.t1 - z.t0) < 1e-12) {
          sp->pieces.push_back(z);
        } else {
          auto lr = z.split(0.5);
          stack.push_back(lr.second);
          stack.push_back(lr.first);
        }
      }
      for (auto& z : sp->pieces) {
        sp->thick.push_back(z.thickness());
        sp->boxes.push_back(z.box());
      }
      r.curve.sp = sp;
    }
    r.box = r.curve.bbox();
    edges.push_back(r);
  }
  for (int fi = 0; fi < d->n_faces; fi++) {
    const IcamFaceDesc& fd = d->faces[fi];
    Face f;
    f.sense = fd.sense >= 0 ? 1.0 : -1.0;
    f.surf.kind = fd.kind;
    f.surf.f = frame_of(fd.f);
    f.surf.a = fd.a;
    f.surf.b = fd.b;
    if (fd.kind == ICAM_NURBS) {
      auto ns = std::make_shared<NurbsSurf>();
      ns->du = fd.du;
      ns->dv = fd.dv;
      ns->nsu = fd.nsu;
      ns->nsv = fd.nsv;
      const double* br = d->breaks + fd.brk_off;
      ns->ub.assign(br, br + fd.nsu + 1);
      ns->vb.assign(br + fd.nsu + 1, br + fd.nsu + 1 + fd.nsv + 1);
      int np = (fd.du + 1) * (fd.dv + 1);
      for (int a = 0; a < fd.nsu; a++)
        for (int b = 0; b < fd.nsv; b++) {
          Patch pa;
          pa.du = fd.du;
          pa.dv = fd.dv;
          const double* c = d->patches + fd.patch_off + size_t(a * fd.nsv + b) * np * 4;
          for (int k = 0; k < np; k++) pa.pw.push_back({c[4 * k], c[4 * k + 1], c[4 * k + 2], c[4 * k + 3]});
          pa.u0 = ns->ub[a];
          pa.u1 = ns->ub[a + 1];
          pa.v0 = ns->vb[b];
          pa.v1 = ns->vb[b + 1];
          ns->spans.push_back(pa);
        }
      ns->build_tree();
      f.surf.ns = ns;
    }
    std::vector<TPiece> pcs;
    int cur_loop = -1;
    for (int k = 0; k < fd.n_uses; k++) {
      const IcamUseDesc& u = d->uses[fd.first_use + k];
      if (u.loop != cur_loop) {
        f.loops.emplace_back();
        cur_loop = u.loop;
      }
      f.loops.back().push_back({u.edge, u.rev != 0});
      if (u.seam) continue;
      for (int j = 0; j < u.n_pc; j++) {
        TPiece t;
        const double* c = d->pcurves + size_t(u.first_pc + j) * 12;
        for (int i = 0; i < 4; i++)
          for (int q = 0; q < 3; q++) t.c[i][q] = c[3 * i + q];
        pcs.push_back(t);
      }
    }
    std::string e2;
    if (!f.trim.build(pcs, {fd.lo[0], fd.lo[1]}, {fd.hi[0], fd.hi[1]}, {fd.period[0], fd.period[1]}, f.sense > 0, &e2)) {
      if (err) *err = "face " + std::to_string(fi) + ": " + e2;
      return false;
    }
    faces.push_back(std::move(f));
  }
  // solid3.rs:797-834 angle-weighted vertex pseudo-normals
  std::vector<V3> pn(verts.size());
  auto use_tan = [&](std::pair<int, bool> u, double s) {
    return u.second ? -edges[u.first].curve.tangent_at(1.0 - s) : edges[u.first].curve.tangent_at(s);
  };
  auto use_end = [&](std::pair<int, bool> u) { return u.second ? edges[u.first].v[0] : edges[u.first].v[1]; };
  for (auto& f : faces)
    for (auto& lp : f.loops)
      for (size_t i = 0; i < lp.size(); i++) {
        auto a = lp[i], b = lp[(i + 1) % lp.size()];
        int v = use_end(a);
        V3 n = f.normal(verts[v].p);
        auto proj = [&](V3 t) { return (t - n * n.dot(t)).unit(); };
        V3 ti = proj(use_tan(a, 1.0)), to = proj(use_tan(b, 0.0));
        double turn = std::atan2(n.dot(ti.cross(to)), ti.dot(to));
        pn[v] = pn[v] + n * (PI - turn);
      }
  for (size_t i = 0; i < verts.size(); i++) verts[i].pn = pn[i];
  std::vector<Box> boxes;
  bbox = empty_box();
  for (auto& f : faces) {
    Box b = face_box(f, edges);
    boxes.push_back(b);
    grow(bbox, b.first);
    grow(bbox, b.second);
  }
  for (auto& e : edges) boxes.push_back(e.box);
  for (auto& v : verts) boxes.push_back({v.p, v.p});
  // solid3.rs:1609-1614, surface3.rs:1418-1440 c0_lines: a B-spline face's interior knot
  // lines where its spans' normals differ (sampled at five points a span), each with its
  // pieces (the after span's side on the line) and the spans either side
  for (size_t fi = 0; fi < faces.size(); fi++) {
    const Face& f = faces[fi];
    if (f.surf.kind != NURBS || !f.surf.ns) continue;
    const NurbsSurf& ns = *f.surf.ns;
    auto unit_n = [](const Patch& pa, double s, double t) {
      SEval e = pa.eval(s, t);
      return e.ps.cross(e.pt).unit();
    };
    for (int k = 0; k < 2; k++) {
      const int na = k == 0 ? ns.nsu : ns.nsv, nb = k == 0 ? ns.nsv : ns.nsu;
      for (int a = 1; a < na; a++) {
        bool crease = false;
        for (int b = 0; b < nb && !crease; b++) {
          const Patch& pb = k == 0 ? ns.span(a - 1, b) : ns.span(b, a - 1);
          const Patch& pn = k == 0 ? ns.span(a, b) : ns.span(b, a);
          for (double t : {0.0, 0.25, 0.5, 0.75, 1.0}) {
            V3 n0 = k == 0 ? unit_n(pb, 1.0, t) : unit_n(pb, t, 1.0);
            V3 n1 = k == 0 ? unit_n(pn, 0.0, t) : unit_n(pn, t, 0.0);
            if ((n0 - n1).len() > 1e-7) crease = true;
          }
        }
        if (!crease) continue;
        C0Line l;
        l.face = int(fi);
        l.k = k;
        l.value = k == 0 ? ns.ub[a] : ns.vb[a];
        for (int b = 0; b < nb; b++) {
          const Patch& pb = k == 0 ? ns.span(a - 1, b) : ns.span(b, a - 1);
          const Patch& pn = k == 0 ? ns.span(a, b) : ns.span(b, a);
          Bez3 z;
          if (k == 0) {
            for (int j = 0; j <= pn.dv; j++) z.pw.push_back(pn.at(0, j));
            z.t0 = pn.v0, z.t1 = pn.v1;
          } else {
            for (int i = 0; i <= pn.du; i++) z.pw.push_back(pn.at(i, 0));
            z.t0 = pn.u0, z.t1 = pn.u1;
          }
          l.pieces.push_back(z);
          l.before.push_back(&pb);
          l.after.push_back(&pn);
        }
        lines.push_back(std::move(l));
      }
    }
  }
  for (auto& l : lines) {
    Box b = empty_box();
    for (auto& z : l.pieces) {
      Box zb = z.box();
      grow(b, zb.first);
      grow(b, zb.second);
    }
    boxes.push_back(b);
  }
  // solid3.rs:1615-1625 poles: each side of a B-spline face's domain that its surface
  // collapses on to one point (surface3.rs:1392-1413 collapsed_sides, 17 points along the
  // side within 1e-12 of the surface's size) is a crease of its search; where the point is
  // at no vertex and the side's middle is inside the face, a point feature with the fan
  // pseudo-normal
  poles.clear();
  for (size_t fi = 0; fi < faces.size(); fi++) {
    Face& f = faces[fi];
    if (f.surf.kind != NURBS || !f.surf.ns) continue;
    NurbsSurf& ns = *f.surf.ns;
    Box sb = ns.bbox();
    double scale = std::max((sb.second - sb.first).len(), 1e-9);
    for (int k = 0; k < 2; k++) {
      const std::vector<double>& rb = k == 0 ? ns.ub : ns.vb;
      const std::vector<double>& ob = k == 0 ? ns.vb : ns.ub;
      const double o0 = ob.front(), o1 = ob.back();
      for (double side : {rb.front(), rb.back()}) {
        auto at = [&](double w) { return k == 0 ? ns.eval(side, w) : ns.eval(w, side); };
        V3 x = at(o0).p;
        bool collapsed = true;
        for (int i = 1; i <= 16 && collapsed; i++)
          if ((at(o0 + (o1 - o0) * i / 16.0).p - x).len() > 1e-12 * scale) collapsed = false;
        if (!collapsed) continue;
        (k == 0 ? ns.cu : ns.cv).push_back(side);
        bool at_vertex = false;
        for (auto& v : verts)
          if ((v.p - x).len() <= tol) at_vertex = true;
        if (at_vertex) continue;
        const double mid = 0.5 * (o0 + o1);
        if (!(k == 0 ? f.trim.inside(side, mid) : f.trim.inside(mid, side))) continue;
        // solid3.rs:1960-1986 fan_normal: near the point the surface is the cone of its
        // limiting tangents S_k(w) with limiting normals S_k x S_kw (u held) or
        // S_kw x S_v (v held), oriented as S_u x S_v just inside; each pair of
        // neighbouring samples whose side is covered by the face adds its mean normal
        // times the angle its tangent turns through
        const double h = side == rb.front() ? 1.0 : -1.0;
        const double step = 1e-9 * (rb.back() - rb.front()) * h;
        const int n = 512;
        V3 out, ptan, pnrm;
        bool have = false, pcov = false;
        for (int i = 0; i <= n; i++) {
          const double w = o0 + (o1 - o0) * i / double(n);
          SEval e = at(w);
          V3 tan = (k == 0 ? e.ps : e.pt) * h;
          V3 nrm = (k == 0 ? e.ps.cross(e.pst) : e.pst.cross(e.pt)) * h;
          const bool cov = k == 0 ? f.trim.inside(side + step, w) : f.trim.inside(w, side + step);
          if (have && pcov && cov && tan.len() > 0.0 && ptan.len() > 0.0) {
            V3 a = ptan.unit(), c = tan.unit();
            const double ang = std::atan2(a.cross(c).len(), a.dot(c));
            V3 m = pnrm.unit() + nrm.unit();
            if (m.len() > 0.0) out = out + m.unit() * ang;
          }
          ptan = tan, pnrm = nrm, pcov = cov, have = true;
        }
        poles.push_back({int(fi), x, out * f.sense});
      }
    }
  }
  for (auto& pl : poles) boxes.push_back({pl.x, pl.x});
  tree_.init(boxes);
  return true;
}

// Bernstein coefficients of degree m times those of degree n (degree m + n).
static std::vector<double> bern_mul(const std::vector<double>& a, const std::vector<double>& b) {
  const int m = int(a.size()) - 1, n = int(b.size()) - 1;
  auto binom = [](int N, int K) {
    double r = 1.0;
    for (int i = 1; i <= K; i++) r = r * (N - K + i) / i;
    return r;
  };
  std::vector<double> c(m + n + 1, 0.0);
  for (int i = 0; i <= m; i++)
    for (int j = 0; j <= n; j++) c[i + j] += binom(m, i) * binom(n, j) / binom(m + n, i + j) * a[i] * b[j];
  return c;
}
static std::vector<double> bern_d(const std::vector<double>& a) {
  const int m = int(a.size()) - 1;
  std::vector<double> d(std::max(m, 1), 0.0);
  for (int i = 0; i < m; i++) d[i] = m * (a[i + 1] - a[i]);
  return d;
}

// surface3.rs:734-757 curve_no_critical_point: the rational curve has no point whose
// chord to p is perpendicular to it (the numerator of d/ds |C - p|^2, in Bernstein form,
// keeps one sign).
static bool curve_no_critical_point(const std::vector<H4>& pw, V3 p) {
  std::vector<double> w, q[3];
  for (auto& h : pw) {
    if (!(h[3] > 0.0)) return false;
    w.push_back(h[3]);
    q[0].push_back(h[0] - p.x * h[3]);
    q[1].push_back(h[1] - p.y * h[3]);
    q[2].push_back(h[2] - p.z * h[3]);
  }
  std::vector<double> qu[3] = {bern_d(q[0]), bern_d(q[1]), bern_d(q[2])};
  auto dot = [](const std::vector<double>* x, const std::vector<double>* y) {
    std::vector<double> s = bern_mul(x[0], y[0]);
    for (int k = 1; k < 3; k++) {
      std::vector<double> t = bern_mul(x[k], y[k]);
      for (size_t i = 0; i < s.size(); i++) s[i] += t[i];
    }
    return s;
  };
  std::vector<double> f = bern_mul(w, dot(q, qu)), g = bern_mul(bern_d(w), dot(q, q));
  for (size_t i = 0; i < f.size(); i++) f[i] -= g[i];
  auto max_abs = [](const std::vector<double>& x) {
    double m = 0.0;
    for (double y : x) m = std::max(m, std::fabs(y));
    return m;
  };
  double q0 = std::max(max_abs(q[0]), std::max(max_abs(q[1]), max_abs(q[2])));
  double q1 = std::max(max_abs(qu[0]), std::max(max_abs(qu[1]), max_abs(qu[2])));
  double size = max_abs(w) * 3.0 * q0 * q1 + max_abs(bern_d(w)) * 3.0 * q0 * q0;
  double lo = INF, hi = -INF;
  for (double x : f) lo = std::min(lo, x), hi = std::max(hi, x);
  return lo > 1e-11 * size || hi < -1e-11 * size;
}

// solid3.rs:1821-1886 c0_line: the nearest point of a knot line inside its face below
// `cutoff` where the distance along the line is critical (where the line meets the face's
// boundary the edges answer): its distance, the point, and the two sides' outward normals
// summed (the span before the line at its far side, the span after at its near side).
bool Exact::c0_line(const C0Line& l, V3 p, double cutoff, ExactStats* st, double* d_out, V3* q_out,
                    V3* n_out) const {
  const Face& f = faces[l.face];
  auto at = [&](double w) { return l.k == 0 ? P2{l.value, w} : P2{w, l.value}; };
  struct E {
    double lb;
    size_t i;
    Bez3 z;
    int depth;
  };
  std::vector<E> heap;
  for (size_t i = 0; i < l.pieces.size(); i++) {
    double lb = box_dist(p, l.pieces[i].box());
    if (lb < cutoff) heap.push_back({lb, i, l.pieces[i], 0});
  }
  double bound = cutoff;
  bool have = false;
  double bd = 0.0, bw = 0.0;
  V3 bq;
  size_t bi = 0;
  int pops = 0;
  while (!heap.empty()) {
    size_t k = 0;
    for (size_t j = 1; j < heap.size(); j++)
      if (heap[j].lb < heap[k].lb) k = j;
    E e = heap[k];
    heap[k] = heap.back();
    heap.pop_back();
    if (e.lb >= bound - DIST_EPS) break;
    if (++pops > 4096) {
      st->capped = true;
      break;
    }
    P2 a = at(e.z.t0), b = at(e.z.t1);
    int state = f.trim.box_class({std::min(a[0], b[0]), std::min(a[1], b[1])}, {std::max(a[0], b[0]), std::max(a[1], b[1])});
    if (state == 0) continue;
    double s = e.z.newton(p, 0.5);
    Eval3 ev = e.z.eval(s);
    double d = (ev.p - p).len();
    double w = e.z.t0 + s * (e.z.t1 - e.z.t0);
    P2 uv = at(w);
    if (d < bound && (state == 1 || f.trim.inside(uv[0], uv[1]))) {
      bound = d;
      V3 r = ev.p - p;
      auto big = [](V3 x) { return std::max(std::fabs(x.x), std::max(std::fabs(x.y), std::fabs(x.z))); };
      double round = 1024.0 * 2.220446049250313e-16 * (big(ev.p) + big(p) + d);
      if (std::fabs(r.dot(ev.d1)) <= (round + 1e-12 * ev.d1.len()) * ev.d1.len()) {
        have = true;
        bd = d, bq = ev.p, bi = e.i, bw = w;
      }
    }
    if (e.depth >= 40 || curve_no_critical_point(e.z.pw, p)) continue;
    auto lr = e.z.split(0.5);
    for (const Bez3* c : {&lr.first, &lr.second}) {
      double lbc = box_dist(p, c->box());
      if (lbc < bound - DIST_EPS) heap.push_back({lbc, e.i, *c, e.depth + 1});
    }
  }
  st->pops += pops;
  if (!have) return false;
  auto side_n = [&](const Patch* pa, double side) {
    double s, t;
    if (l.k == 0)
      s = side, t = (bw - pa->v0) / (pa->v1 - pa->v0);
    else
      s = (bw - pa->u0) / (pa->u1 - pa->u0), t = side;
    SEval e = pa->eval(s, t);
    return e.ps.cross(e.pt).unit();
  };
  *n_out = (side_n(l.before[bi], 1.0) + side_n(l.after[bi], 0.0)) * f.sense;
  *d_out = bd;
  *q_out = bq;
  return true;
}

// solid3.rs:1891-1897 normal_at
V3 Exact::normal_at(size_t fi, V3 x) const {
  const Face& f = faces[fi];
  if (f.surf.kind == NURBS) {
    SurfHit h;
    if (f.surf.ns->closest(x, 4.0 * tol + 1e-9, &h) || f.surf.ns->closest(x, INF, &h)) return h.n * f.sense;
    return V3(0, 0, 1) * f.sense;
  }
  return f.normal(x);
}

// solid3.rs:1901-1945 face (certified loops on every face of these descriptions)
bool Exact::face(size_t fi, V3 p, double cutoff, ExactStats* st, double* d, V3* q, V3* n) const {
  const Face& f = faces[fi];
  if (f.surf.kind == NURBS) {
    SurfHit h;
    bool complete = true;
    int pops = 0;
    bool have = f.surf.ns->closest_trimmed(p, cutoff, &f.trim, &h, &complete, &pops);
    st->pops += pops;
    st->capped |= !complete;
    if (!have) return false;
    if (!(h.dist < cutoff && h.n.len() > 0.5)) return false;
    *d = h.dist;
    *q = h.q;
    *n = h.n * f.sense;
    return true;
  }
  V3 x = f.surf.foot(p);
  double dd = (p - x).len();
  if (!(dd < cutoff)) return false;
  // A cone's apex is a singular foot: the edges and vertices answer there
  // (solid3.rs:1919-1924; no synthetic face holds an apex or a torus tip).
  if (f.surf.kind == CONE) {
    V3 apex = f.surf.f.o + f.surf.f.z * (-f.surf.a / std::tan(f.surf.b));
    if ((apex - x).len() <= 1e-12 * (1.0 + apex.len())) return false;
  }
  double u, v;
  f.surf.uv(x, &u, &v);
  if (!f.trim.inside(u, v)) return false;
  *d = dd;
  *q = x;
  *n = f.normal(x);
  return true;
}

// solid3.rs:1758-1816 sdf_within
Sd Exact::sdf_within(V3 p, double bound, ExactStats* st) const {
  ExactStats local;
  if (!st) st = &local;
  *st = ExactStats();
  size_t nF = nf(), nE = ne();
  Sd best{bound, p, 2, 0, false};
  bool found = false;
  auto sign = [](double x) { return x < 0.0 ? -1.0 : 1.0; };
  bool cusp = false;
  tree_.nearest_first(p, bound, [&](size_t id) {
    st->features++;
    double cur = std::fabs(best.d);
    double before = best.d;
    if (id < nF) {
      double d;
      V3 q, n;
      if (face(id, p, cur, st, &d, &q, &n)) best = {d * sign((p - q).dot(n)), q, 0, int(id), false};
    } else if (id < nF + nE) {
      size_t ei = id - nF;
      const EdgeRec& e = edges[ei];
      Foot3 c;
      if (e.curve.closest_below(p, cur, &c) && c.near == INTERIOR) {
        V3 pn = normal_at(e.faces[0], c.q) + normal_at(e.faces[1], c.q);
        best = {c.dist * sign((p - c.q).dot(pn)), c.q, 1, int(ei), false};
        cusp = pn.len() < 1e-9;
      }
    } else if (id < nF + nE + verts.size()) {
      size_t vi = id - nF - nE;
      const Vert& v = verts[vi];
      double d = (p - v.p).len();
      if (d < cur) best = {d * sign((p - v.p).dot(v.pn)), v.p, 2, int(vi), false};
    } else if (id < nF + nE + verts.size() + lines.size()) {  // solid3.rs:1790-1795 a knot line
      const C0Line& l = lines[id - nF - nE - verts.size()];
      double d;
      V3 q, n;
      if (c0_line(l, p, cur, st, &d, &q, &n)) best = {d * sign((p - q).dot(n)), q, 0, l.face, false};
    } else {  // solid3.rs:1795-1801 a pole
      const Pole& pl = poles[id - nF - nE - verts.size() - lines.size()];
      double d = (p - pl.x).len();
      if (d < cur) best = {d * sign((p - pl.x).dot(pl.n)), pl.x, 0, pl.face, false};
    }
    if (best.d != before) {
      found = true;
      if (best.kind != 1) cusp = false;
    }
    return std::fabs(best.d);
  });
  if (!found && std::isfinite(bound)) return sdf_within(p, INF, st);
  st->cusp = cusp;
  best.unsure = st->capped || st->cusp;
  return best;
}

// solid3.rs:1661-1690 candidates
std::vector<size_t> Exact::candidates(V3 c, double r, double d) const {
  size_t nF = nf(), nE = ne();
  double reach = d + 2.0 * r;
  std::vector<size_t> out;
  tree_.visit(Box{c, c}, reach, [&](size_t id) {
    double lb;
    if (id < nF) {
      double b = box_dist(c, tree_.boxes_of(id));
      lb = faces[id].surf.kind == NURBS ? b : std::max((c - faces[id].surf.foot(c)).len(), b);
    } else if (id < nF + nE) {
      const Edge3& e = edges[id - nF].curve;
      lb = e.kind <= 1 ? e.closest(c).dist : 0.0;
    } else if (id < nF + nE + verts.size()) {
      lb = (c - verts[id - nF - nE].p).len();
    } else if (id >= nF + nE + verts.size() + lines.size()) {
      lb = (c - poles[id - nF - nE - verts.size() - lines.size()].x).len();
    } else {
      lb = box_dist(c, tree_.boxes_of(id));
    }
    if (lb <= reach) out.push_back(id);
  });
  return out;
}

// solid3.rs:1710-1724 kind_of: analytic face 0, B-spline face 1, line/arc edge 2,
// other edge 3, vertex 4
int Exact::kind_of(size_t id) const {
  if (id < nf()) return faces[id].surf.kind == NURBS ? 1 : 0;
  if (id < nf() + ne()) return edges[id - nf()].curve.kind <= 1 ? 2 : 3;
  if (id < nf() + ne() + nv()) return 4;
  if (id < nf() + ne() + nv() + lines.size()) return 3;  // a knot line: as a spline edge
  return 4;                                              // a pole: as a vertex
}

// partcache.rs:962-970 packed
int packed_kind(const int16_t* q) {
  bool all_pos = true, all_nonpos = true;
  for (int n = 0; n < 729; n++) {
    if (!(q[n] > 0)) all_pos = false;
    if (!(q[n] <= 0)) all_nonpos = false;
  }
  if (all_pos) return 1;
  if (all_nonpos) return 2;
  return 0;
}

void pack_words(const int16_t* q, uint32_t* w) {
  for (int k = 0; k < 365; k++) {
    uint32_t lo = uint16_t(q[2 * k]);
    uint32_t hi = 2 * k + 1 < 729 ? uint32_t(uint16_t(q[2 * k + 1])) << 16 : 0u;
    w[k] = lo | hi;
  }
}

}  // namespace oracle
