// Builds the device layout of a solid (pack.h) from its description (icam_solid.h):
// trim trees per face, B-spline spans raised to bicubic and split into sub-patches
// that certify convexity for the pack's `need`, flat spline-edge pieces with their
// bounds, angle-weighted vertex pseudo-normals, and one bounding-volume tree over
// every feature. Host code; the arrays are uploaded by the caller.
#include "pack_build.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace icam {

namespace {

const double PI = 3.14159265358979323846;

V vec(const double* x) { return V(x[0], x[1], x[2]); }

struct Axial {
  double theta, rho, h;
  V er;
};
Axial axial(const DFace& f, V p) {
  V d = p - vec(f.o);
  V x = vec(f.x), y = vec(f.y), z = vec(f.z);
  double lx = d.dot(x), ly = d.dot(y), lz = d.dot(z);
  double rho = std::sqrt(lx * lx + ly * ly);
  double th = rho > 0 ? std::atan2(ly, lx) : 0.0;
  return {th, rho, lz, x * std::cos(th) + y * std::sin(th)};
}

// Outward normal of an analytic face at a point on it (surface3.rs:132-148 times the sense).
V analytic_normal(const DFace& f, V q) {
  V n;
  switch (f.kind) {
    case S_PLANE: n = vec(f.z); break;
    case S_CYLINDER: n = axial(f, q).er; break;
    case S_CONE: n = axial(f, q).er * std::cos(f.b) - vec(f.z) * std::sin(f.b); break;
    case S_SPHERE: n = (q - vec(f.o)).unit(); break;
    default: n = (q - (vec(f.o) + axial(f, q).er * f.a)).unit(); break;
  }
  return n * f.sense;
}

// The nearest point of a B-spline face's spans to a point on (or very near) it: Newton
// from each span's middle, kept in its span; returns (u, v) and the unit normal Su x Sv.
struct SpanGrid {
  std::vector<Bicubic> spans;
  int nsu, nsv;
};
// The face's domain, from its spans: u in [u0, u1], v in [v0, v1].
void grid_domain(const SpanGrid& g, double* u0, double* u1, double* v0, double* v1) {
  *u0 = g.spans.front().u0, *v0 = g.spans.front().v0;
  *u1 = g.spans[size_t(g.nsu - 1) * g.nsv].u1, *v1 = g.spans[size_t(g.nsv - 1)].v1;
}

// The surface at global (u, v), with its derivatives along the span's own parameters.
void grid_eval(const SpanGrid& g, double u, double v, V* P, V* Ps, V* Pt, V* Pst) {
  int a = 0, b = 0;
  while (a + 1 < g.nsu && g.spans[size_t(a + 1) * g.nsv].u0 <= u) a++;
  while (b + 1 < g.nsv && g.spans[size_t(b + 1)].v0 <= v) b++;
  const Bicubic& sp = g.spans[size_t(a) * g.nsv + b];
  const double s = std::min(std::max((u - sp.u0) / (sp.u1 - sp.u0), 0.0), 1.0);
  const double t = std::min(std::max((v - sp.v0) / (sp.v1 - sp.v0), 0.0), 1.0);
  V Pss, Ptt;
  sp.eval(s, t, P, Ps, Pt, &Pss, Pst, &Ptt);
}

// A side of a B-spline face's domain that its surface collapses on to one point (a
// pole's side): k 0 when u is held (at `value`), the point x.
struct Collapsed {
  int k;
  double value;
  V x;
};

// surface3.rs:1392-1413 collapsed_sides: the domain sides along which 17 evenly spaced
// points of the surface lie within 1e-12 of its control box's diagonal of the first.
std::vector<Collapsed> collapsed_sides(const SpanGrid& g) {
  Bx bx;
  for (auto& sp : g.spans) bx.add(sp.box());
  const double scale = std::max((bx.hi - bx.lo).len(), 1e-9);
  double u0, u1, v0, v1;
  grid_domain(g, &u0, &u1, &v0, &v1);
  std::vector<Collapsed> out;
  for (int k = 0; k < 2; k++) {
    const double o0 = k == 0 ? v0 : u0, o1 = k == 0 ? v1 : u1;
    for (double side : k == 0 ? std::vector<double>{u0, u1} : std::vector<double>{v0, v1}) {
      auto at = [&](double w) {
        V P, Ps, Pt, Pst;
        if (k == 0)
          grid_eval(g, side, w, &P, &Ps, &Pt, &Pst);
        else
          grid_eval(g, w, side, &P, &Ps, &Pt, &Pst);
        return P;
      };
      const V x = at(o0);
      bool same = true;
      for (int i = 1; i <= 16 && same; i++)
        if ((at(o0 + (o1 - o0) * i / 16.0) - x).len() > 1e-12 * scale) same = false;
      if (same) out.push_back({k, side, x});
    }
  }
  return out;
}

// Whether local (s0, t0) of span (a, b) lies on one of the face's collapsed sides.
bool on_collapsed(const SpanGrid& g, const std::vector<Collapsed>& cs, int a, int b, double s0, double t0) {
  const Bicubic& sp = g.spans[size_t(a) * g.nsv + b];
  const double u = s0 == 0.0 ? sp.u0 : (s0 == 1.0 ? sp.u1 : sp.u0 + s0 * (sp.u1 - sp.u0));
  const double v = t0 == 0.0 ? sp.v0 : (t0 == 1.0 ? sp.v1 : sp.v0 + t0 * (sp.v1 - sp.v0));
  for (auto& c : cs)
    if ((c.k == 0 ? u : v) == c.value) return true;
  return false;
}

// A B-spline face's creases: the interior span boundaries across which the spans' unit
// normals differ (sampled at five points a span; 1e-7), where the surface is only C0 and
// folds (Exact::c0_line, solid3.rs:1821; the reference finds them by knots of full
// multiplicity, a knot line with a continuous normal needs no feature of its own). Each
// (k, a): the boundary before span a along u (k 0) or v (k 1). Samples on a collapsed
// side (a pole's, where the normal is not defined) are skipped. False, with the reason,
// when the normal vanishes anywhere else on a span's side: a degenerate point that no
// feature of this pack covers.
bool span_creases(const SpanGrid& g, const std::vector<Collapsed>& cs, std::vector<std::pair<int, int>>* creases,
                  std::string* why) {
  auto normal = [](const Bicubic& sp, double s, double t, double* len) {
    V P, Ps, Pt, Pss, Pst, Ptt;
    sp.eval(s, t, &P, &Ps, &Pt, &Pss, &Pst, &Ptt);
    V n = Ps.cross(Pt);
    *len = n.len() / std::max(Ps.len() * Pt.len(), 1e-300);
    return n.unit();
  };
  const double ts[5] = {0.0, 0.25, 0.5, 0.75, 1.0};
  for (int a = 0; a < g.nsu; a++)
    for (int b = 0; b < g.nsv; b++)
      for (double t : ts)
        for (int side = 0; side < 4; side++) {
          const double s0 = side == 0 ? 0.0 : (side == 1 ? 1.0 : t), t0 = side == 2 ? 0.0 : (side == 3 ? 1.0 : t);
          if (on_collapsed(g, cs, a, b, s0, t0)) continue;
          double l;
          normal(g.spans[size_t(a) * g.nsv + b], s0, t0, &l);
          if (!(l > 1e-9)) {
            *why = "its B-spline surface has no normal at a point off its collapsed sides: not packed";
            return false;
          }
        }
  for (int k = 0; k < 2; k++) {
    const int na = k == 0 ? g.nsu : g.nsv, nb = k == 0 ? g.nsv : g.nsu;
    for (int a = 1; a < na; a++) {
      bool crease = false;
      for (int b = 0; b < nb && !crease; b++) {
        const Bicubic& p0 = g.spans[k == 0 ? (a - 1) * g.nsv + b : b * g.nsv + a - 1];
        const Bicubic& p1 = g.spans[k == 0 ? a * g.nsv + b : b * g.nsv + a];
        for (double t : ts) {
          if (k == 0 ? on_collapsed(g, cs, a, b, 0.0, t) : on_collapsed(g, cs, b, a, t, 0.0)) continue;
          double l0, l1;
          const V n0 = k == 0 ? normal(p0, 1.0, t, &l0) : normal(p0, t, 1.0, &l0);
          const V n1 = k == 0 ? normal(p1, 0.0, t, &l1) : normal(p1, t, 0.0, &l1);
          if ((n0 - n1).len() > 1e-7) crease = true;
        }
      }
      if (crease) creases->push_back({k, a});
    }
  }
  return true;
}

// A rational cubic with its parameter range on the curve it was cut from.
struct CutPiece {
  Cubic3 z;
  double t0, t1;
};

// A spline curve's pieces made flat (split until the control polygon turns <= 0.35,
// curve3.rs:1017-1031), then each halved (up to 5 times) until |C - p|^2 certifies
// convex for every p within `need` of it, so that points that near take one Newton
// solve instead of the subdivision search; the curve and its closest points are the
// same, the halves' ends only add points of it to try.
std::vector<CutPiece> flat_pieces(const std::vector<CutPiece>& in, double need) {
  std::vector<CutPiece> flat, stack(in.rbegin(), in.rend());
  while (!stack.empty()) {
    CutPiece q = stack.back();
    stack.pop_back();
    if (q.z.turning() <= 0.35 || flat.size() > 100000) {
      flat.push_back(q);
    } else {
      CutPiece l, r;
      q.z.split(0.5, &l.z, &r.z);
      const double m = 0.5 * (q.t0 + q.t1);
      l.t0 = q.t0, l.t1 = m, r.t0 = m, r.t1 = q.t1;
      stack.push_back(r);
      stack.push_back(l);
    }
  }
  std::vector<CutPiece> fine;
  std::vector<std::pair<CutPiece, int>> st;
  for (const CutPiece& z0 : flat) {
    st.assign(1, {z0, 0});
    while (!st.empty()) {
      auto q = st.back();
      st.pop_back();
      if (q.second >= 5 || piece_certifies(q.first.z, need)) {
        fine.push_back(q.first);
      } else {
        CutPiece l, r;
        q.first.z.split(0.5, &l.z, &r.z);
        const double m = 0.5 * (q.first.t0 + q.first.t1);
        l.t0 = q.first.t0, l.t1 = m, r.t0 = m, r.t1 = q.first.t1;
        st.push_back({r, q.second + 1});
        st.push_back({l, q.second + 1});
      }
    }
  }
  return fine;
}

void nearest_on(const SpanGrid& g, V x, double* u, double* v, V* n, double* dist) {
  double best = 1e300;
  for (auto& sp : g.spans) {
    double s = 0.5, t = 0.5;
    for (int it = 0; it < 40; it++) {
      V P, Ps, Pt, Pss, Pst, Ptt;
      sp.eval(s, t, &P, &Ps, &Pt, &Pss, &Pst, &Ptt);
      V r = P - x;
      double g0 = Ps.dot(r), g1 = Pt.dot(r);
      double a = Ps.dot(Ps) + Pss.dot(r), b = Ps.dot(Pt) + Pst.dot(r), c = Pt.dot(Pt) + Ptt.dot(r);
      if (!(a > 0 && a * c - b * b > 0)) a = Ps.dot(Ps), b = Ps.dot(Pt), c = Pt.dot(Pt);
      double det = a * c - b * b;
      if (std::fabs(det) < 1e-300) break;
      double ds = -(c * g0 - b * g1) / det, dt = -(a * g1 - b * g0) / det;
      double ns = std::min(std::max(s + ds, 0.0), 1.0), nt = std::min(std::max(t + dt, 0.0), 1.0);
      double moved = std::fabs(ns - s) + std::fabs(nt - t);
      s = ns, t = nt;
      if (moved < 1e-15) break;
    }
    V P, Ps, Pt;
    sp.eval(s, t, &P, &Ps, &Pt, nullptr, nullptr, nullptr);
    double d = (P - x).len();
    if (d < best) {
      best = d;
      *u = sp.u0 + s * (sp.u1 - sp.u0);
      *v = sp.v0 + t * (sp.v1 - sp.v0);
      *n = Ps.cross(Pt).unit();
    }
  }
  *dist = best;
}

struct Item {
  uint32_t code;
  Bx box;
};

// Median split on the longest axis of the centroids' box, into the node at `slot`;
// leaves of at most 4, a node's two children stored side by side.
void build_bvh(std::vector<Item>& items, int a, int b, int slot, std::vector<DBvh>& nodes,
               std::vector<uint32_t>& out_items) {
  Bx bx, cb;
  for (int i = a; i < b; i++) {
    bx.add(items[i].box);
    cb.add(items[i].box.mid());
  }
  for (int k = 0; k < 3; k++) {
    nodes[slot].lo[k] = std::nextafter(float(bx.lo[k]), -INFINITY);
    nodes[slot].hi[k] = std::nextafter(float(bx.hi[k]), INFINITY);
  }
  if (b - a <= 4) {
    nodes[slot].first = int(out_items.size());
    nodes[slot].count = b - a;
    for (int i = a; i < b; i++) out_items.push_back(items[i].code);
    return;
  }
  V ext = cb.hi - cb.lo;
  int ax = ext.x >= ext.y && ext.x >= ext.z ? 0 : (ext.y >= ext.z ? 1 : 2);
  int m = (a + b) / 2;
  std::nth_element(items.begin() + a, items.begin() + m, items.begin() + b,
                   [&](const Item& p, const Item& q) { return p.box.mid()[ax] < q.box.mid()[ax]; });
  int kids = int(nodes.size());
  nodes.resize(kids + 2);
  nodes[slot].first = kids;
  nodes[slot].count = 0;
  build_bvh(items, a, m, kids, nodes, out_items);
  build_bvh(items, m, b, kids + 1, nodes, out_items);
}

}  // namespace

bool build_pack(const IcamSolidDesc* d, double need, HostPack* hp, std::string* err) {
  HostPack& P = *hp;
  P = HostPack();
  P.tol = d->tol;
  // A closed face (a sphere, a torus) has no edges and no vertices: only faces are required.
  if (d->n_faces <= 0 || d->n_edges < 0 || d->n_verts < 0 || (d->n_edges > 0 && !d->edges) ||
      (d->n_verts > 0 && !d->verts)) {
    *err = "empty solid";
    return false;
  }
  // ---------------------------------------------------------------- faces and spans
  std::vector<SpanGrid> grids(d->n_faces);
  std::vector<std::vector<std::pair<int, int>>> creases(d->n_faces);
  std::vector<std::vector<Collapsed>> collapsed(d->n_faces);
  std::vector<TrimTree> trees(d->n_faces);
  for (int fi = 0; fi < d->n_faces; fi++) {
    const IcamFaceDesc& fd = d->faces[fi];
    DFace f{};
    f.kind = fd.kind;
    f.sense = fd.sense >= 0 ? 1.0 : -1.0;
    for (int k = 0; k < 3; k++) {
      f.o[k] = fd.f.o[k];
      f.z[k] = fd.f.z[k];
      f.x[k] = fd.f.x[k];
    }
    V y = vec(f.z).cross(vec(f.x));
    f.y[0] = y.x, f.y[1] = y.y, f.y[2] = y.z;
    f.a = fd.a;
    f.b = fd.b;
    for (int k = 0; k < 2; k++) {
      f.lo[k] = fd.lo[k];
      f.hi[k] = fd.hi[k];
      f.period[k] = fd.period[k];
    }
    f.nurbs = -1;
    if (fd.kind == ICAM_NURBS) {
      if (fd.du < 1 || fd.du > 3 || fd.dv < 1 || fd.dv > 3) {
        *err = "face " + std::to_string(fi) + ": B-spline degrees above 3 are not packed";
        return false;
      }
      DNurbs nb{};
      nb.face = fi;
      nb.first_span = int(P.span_cp.size() / 16);
      nb.nsu = fd.nsu;
      nb.nsv = fd.nsv;
      nb.first_break = int(P.breaks.size());
      const double* br = d->breaks + fd.brk_off;
      for (int k = 0; k <= fd.nsu + fd.nsv + 1; k++) P.breaks.push_back(br[k]);
      int np = (fd.du + 1) * (fd.dv + 1);
      grids[fi].nsu = fd.nsu;
      grids[fi].nsv = fd.nsv;
      for (int a = 0; a < fd.nsu; a++)
        for (int b = 0; b < fd.nsv; b++) {
          const double* c = d->patches + fd.patch_off + size_t(a * fd.nsv + b) * np * 4;
          // rows along v raised to cubic, then columns along u
          std::vector<std::vector<H>> rows(fd.du + 1);
          for (int i = 0; i <= fd.du; i++) {
            std::vector<H> r;
            for (int j = 0; j <= fd.dv; j++) r.push_back({c[4 * (i * (fd.dv + 1) + j)], c[4 * (i * (fd.dv + 1) + j) + 1], c[4 * (i * (fd.dv + 1) + j) + 2], c[4 * (i * (fd.dv + 1) + j) + 3]});
            while (r.size() < 4) r = elevate(r);
            rows[i] = r;
          }
          Bicubic bc;
          for (int j = 0; j < 4; j++) {
            std::vector<H> col;
            for (int i = 0; i <= fd.du; i++) col.push_back(rows[i][j]);
            while (col.size() < 4) col = elevate(col);
            for (int i = 0; i < 4; i++) bc.p[i][j] = col[i];
          }
          bc.u0 = br[a];
          bc.u1 = br[a + 1];
          bc.v0 = br[fd.nsu + 1 + b];
          bc.v1 = br[fd.nsu + 1 + b + 1];
          grids[fi].spans.push_back(bc);
          for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
              const H& h = bc.p[i][j];
              P.span_cp.push_back({h[0], h[1], h[2], h[3]});
            }
        }
      std::string why;
      collapsed[fi] = collapsed_sides(grids[fi]);
      if (!span_creases(grids[fi], collapsed[fi], &creases[fi], &why)) {
        *err = "face " + std::to_string(fi) + ": " + why;
        return false;
      }
      f.nurbs = int(P.nurbs.size());
      P.nurbs.push_back(nb);
    } else if (fd.kind < 0 || fd.kind > 4) {
      *err = "face " + std::to_string(fi) + ": unknown surface kind";
      return false;
    }
    // trim loops from the uses' parameter-domain curves (seams are not boundaries)
    std::vector<TP> raw;
    for (int k = 0; k < fd.n_uses; k++) {
      const IcamUseDesc& u = d->uses[fd.first_use + k];
      if (u.seam) continue;
      for (int j = 0; j < u.n_pc; j++) {
        TP t;
        const double* c = d->pcurves + size_t(u.first_pc + j) * 12;
        for (int i = 0; i < 4; i++)
          for (int q = 0; q < 3; q++) t.c[i][q] = c[3 * i + q];
        raw.push_back(t);
      }
    }
    std::string e2;
    if (!trees[fi].build(raw, fd.lo, fd.hi, fd.period, f.sense > 0, &e2)) {
      *err = "face " + std::to_string(fi) + ": " + e2;
      return false;
    }
    const TrimTree& tt = trees[fi];
    if (tt.pieces.empty()) {
      f.trim = -1;
    } else {
      int c0 = int(P.cells.size()), i0 = int(P.insts.size()), p0 = int(P.tpieces.size() / 12);
      for (auto& pc : tt.pieces)
        for (int i = 0; i < 4; i++)
          for (int q = 0; q < 3; q++) P.tpieces.push_back(pc.c[i][q]);
      for (auto& in : tt.inst) P.insts.push_back({p0 + in.first, 0, {in.second[0], in.second[1]}});
      for (auto& c : tt.cells) {
        DCell dc{};
        for (int k = 0; k < 2; k++) {
          dc.lo[k] = c.lo[k];
          dc.hi[k] = c.hi[k];
          dc.r[k] = c.r[k];
        }
        dc.inside = c.inside;
        dc.kind = c.kind;
        if (c.kind == 1) {
          dc.first = int(P.among.size());
          dc.count = int(c.among.size());
          for (int i : c.among) P.among.push_back(i0 + i);
        }
        if (c.kind == 2)
          for (int k = 0; k < 4; k++) dc.kids[k] = c0 + c.kids[k];
        P.cells.push_back(dc);
      }
      f.trim = c0;
    }
    P.faces.push_back(f);
  }
  // ---------------------------------------------------------------- edges
  for (int ei = 0; ei < d->n_edges; ei++) {
    const IcamEdgeDesc& ed = d->edges[ei];
    DEdge e{};
    e.kind = ed.kind;
    e.f0 = ed.f0;
    e.f1 = ed.f1;
    Bx box;
    if (ed.kind == ICAM_EDGE_LINE) {
      for (int k = 0; k < 3; k++) e.a[k] = ed.a[k], e.b[k] = ed.b[k];
      box.add(vec(e.a));
      box.add(vec(e.b));
    } else if (ed.kind == ICAM_EDGE_ARC) {
      for (int k = 0; k < 3; k++) e.o[k] = ed.f.o[k], e.z[k] = ed.f.z[k], e.x[k] = ed.f.x[k];
      V y = vec(e.z).cross(vec(e.x));
      e.y[0] = y.x, e.y[1] = y.y, e.y[2] = y.z;
      e.r = ed.r;
      e.t0 = ed.t0;
      e.sweep = ed.sweep;
      // the whole circle's box (curve3.rs:690-696)
      V axes[3] = {V(1, 0, 0), V(0, 1, 0), V(0, 0, 1)};
      for (V ax : axes) {
        double ex = std::sqrt(std::max(1.0 - std::pow(vec(e.z).dot(ax), 2), 0.0)) * e.r;
        box.add(vec(e.o) + ax * ex);
        box.add(vec(e.o) - ax * ex);
      }
    } else if (ed.kind == ICAM_EDGE_SPLINE) {
      if (ed.degree < 1 || ed.degree > 3) {
        *err = "edge " + std::to_string(ei) + ": spline degrees above 3 are not packed";
        return false;
      }
      std::vector<CutPiece> cut;
      for (int k = 0; k < ed.n_pieces; k++) {
        const double* c = d->cpieces + size_t(ed.first_piece + k) * (ed.degree + 1) * 4;
        std::vector<H> q;
        for (int j = 0; j <= ed.degree; j++) q.push_back({c[4 * j], c[4 * j + 1], c[4 * j + 2], c[4 * j + 3]});
        while (q.size() < 4) q = elevate(q);
        CutPiece z;
        for (int j = 0; j < 4; j++) z.z.c[j] = q[j];
        z.t0 = k, z.t1 = k + 1;
        cut.push_back(z);
      }
      std::vector<CutPiece> fp = flat_pieces(cut, need);
      std::vector<Cubic3> flat;
      for (auto& q : fp) flat.push_back(q.z);
      e.first_piece = int(P.pieces.size());
      e.n_pieces = int(flat.size());
      for (size_t k = 0; k < flat.size(); k++) {
        DPiece pc{};
        pc.edge = ei;
        pc.first = k == 0;
        pc.last = k + 1 == flat.size();
        for (int j = 0; j < 4; j++)
          for (int c = 0; c < 4; c++) pc.cp[j][c] = flat[k].c[j][c];
        Bx pb = flat[k].box();
        for (int c = 0; c < 3; c++) pc.box[c] = pb.lo[c], pc.box[3 + c] = pb.hi[c];
        box.add(pb);
        pc.thick = flat[k].thickness();
        if (!piece_bounds(flat[k].c, &pc.lam, pc.d2)) {
          *err = "edge " + std::to_string(ei) + ": a weight is not positive";
          return false;
        }
        for (int side = 0; side < 2; side++) {
          int fi = side == 0 ? ed.f0 : ed.f1;
          for (int end = 0; end < 2; end++) pc.uv[side][end][0] = pc.uv[side][end][1] = -1e300;
          if (fi < 0 || d->faces[fi].kind != ICAM_NURBS) continue;
          for (int end = 0; end < 2; end++) {
            double u, v, dist;
            V n;
            nearest_on(grids[fi], hv(flat[k].c[end * 3]), &u, &v, &n, &dist);
            pc.uv[side][end][0] = u;
            pc.uv[side][end][1] = v;
          }
        }
        P.pieces.push_back(pc);
      }
    } else {
      *err = "edge " + std::to_string(ei) + ": unknown curve kind";
      return false;
    }
    if (ed.kind != ICAM_EDGE_SPLINE)
      for (int side = 0; side < 2; side++) {
        int fi = side == 0 ? ed.f0 : ed.f1;
        if (fi >= 0 && d->faces[fi].kind == ICAM_NURBS) {
          *err = "edge " + std::to_string(ei) + ": a line or arc edge of a B-spline face is not packed";
          return false;
        }
      }
    for (int c = 0; c < 3; c++) e.box[c] = box.lo[c], e.box[3 + c] = box.hi[c];
    P.edges.push_back(e);
  }
  // ---------------------------------------------------------------- creases (solid3.rs:1821-1886)
  // A B-spline face's crease as an edge of that face with itself: its pieces are the
  // iso-curve on the knot line (the side of the span after it), flat and certified as a
  // spline edge's; each piece keeps the parameters of its ends on either side, nudged a
  // billionth of a span into the span before the line for side 0, so that the normals
  // summed for its sign are the two spans' (the span before at its far side, the span
  // after at its near side); its first and last pieces' outer ends are where the line
  // meets the face's boundary, which the boundary's edges answer. A crease must lie
  // wholly inside its face's loops (the device does not test a crease's feet against
  // them); one crossing them is refused.
  for (int fi = 0; fi < d->n_faces; fi++) {
    if (creases[fi].empty()) continue;
    const SpanGrid& g = grids[fi];
    const DNurbs& nbr = P.nurbs[P.faces[fi].nurbs];
    const double* ubr = P.breaks.data() + nbr.first_break;
    const double* vbr = ubr + g.nsu + 1;
    for (auto [k, a] : creases[fi]) {
      const double value = k == 0 ? ubr[a] : vbr[a];
      const double* other = k == 0 ? vbr : ubr;
      const int no = k == 0 ? g.nsv : g.nsu;
      const double eo = 1e-9 * (other[no] - other[0]);
      double lo[2], hi[2];
      lo[k] = hi[k] = value;
      lo[1 - k] = other[0] + eo;
      hi[1 - k] = other[no] - eo;
      if (trees[fi].box_class(lo, hi) != 1) {
        *err = "face " + std::to_string(fi) + ": a crease that crosses its face's loops is not packed";
        return false;
      }
      std::vector<CutPiece> cut;
      for (int b = 0; b < no; b++) {
        const Bicubic& sp = g.spans[k == 0 ? a * g.nsv + b : b * g.nsv + a];
        CutPiece z;
        for (int j = 0; j < 4; j++) z.z.c[j] = k == 0 ? sp.p[0][j] : sp.p[j][0];
        z.t0 = other[b], z.t1 = other[b + 1];
        cut.push_back(z);
      }
      std::vector<CutPiece> fp = flat_pieces(cut, need);
      const double span_w = k == 0 ? ubr[a] - ubr[a - 1] : vbr[a] - vbr[a - 1];
      DEdge e{};
      e.kind = 3;  // a crease
      e.f0 = e.f1 = fi;
      e.first_piece = int(P.pieces.size());
      e.n_pieces = int(fp.size());
      Bx box;
      for (size_t q = 0; q < fp.size(); q++) {
        DPiece pc{};
        pc.edge = int(P.edges.size());
        pc.first = q == 0;
        pc.last = q + 1 == fp.size();
        for (int j = 0; j < 4; j++)
          for (int c = 0; c < 4; c++) pc.cp[j][c] = fp[q].z.c[j][c];
        Bx pb = fp[q].z.box();
        for (int c = 0; c < 3; c++) pc.box[c] = pb.lo[c], pc.box[3 + c] = pb.hi[c];
        box.add(pb);
        pc.thick = fp[q].z.thickness();
        if (!piece_bounds(fp[q].z.c, &pc.lam, pc.d2)) {
          *err = "face " + std::to_string(fi) + ": a weight of a crease is not positive";
          return false;
        }
        for (int side = 0; side < 2; side++)
          for (int end = 0; end < 2; end++) {
            const double held = side == 0 ? value - 1e-9 * span_w : value;
            const double along = end == 0 ? fp[q].t0 : fp[q].t1;
            pc.uv[side][end][k] = held;
            pc.uv[side][end][1 - k] = along;
          }
        P.pieces.push_back(pc);
      }
      for (int c = 0; c < 3; c++) e.box[c] = box.lo[c], e.box[3 + c] = box.hi[c];
      P.edges.push_back(e);
    }
  }
  // ---------------------------------------------------------------- face boxes (solid3.rs:1211-1278)
  for (int fi = 0; fi < d->n_faces; fi++) {
    DFace& f = P.faces[fi];
    const IcamFaceDesc& fd = d->faces[fi];
    Bx bx;
    auto circle_box = [&](V c, V z, double r) {
      V axes[3] = {V(1, 0, 0), V(0, 1, 0), V(0, 0, 1)};
      for (V ax : axes) {
        double e = std::sqrt(std::max(1.0 - std::pow(z.dot(ax), 2), 0.0)) * r;
        bx.add(c + ax * e);
        bx.add(c - ax * e);
      }
    };
    auto edge_box = [&](int ei) {
      Bx b;
      b.add(V(P.edges[ei].box[0], P.edges[ei].box[1], P.edges[ei].box[2]));
      b.add(V(P.edges[ei].box[3], P.edges[ei].box[4], P.edges[ei].box[5]));
      return b;
    };
    if (f.kind == S_PLANE) {
      for (int k = 0; k < fd.n_uses; k++) bx.add(edge_box(d->uses[fd.first_use + k].edge));
    } else if (f.kind == S_CYLINDER || f.kind == S_CONE) {
      double h0 = 1e300, h1 = -1e300;
      for (int k = 0; k < fd.n_uses; k++) {
        Bx eb = edge_box(d->uses[fd.first_use + k].edge);
        for (int q = 0; q < 8; q++) {
          V c((q & 1) ? eb.hi.x : eb.lo.x, (q & 2) ? eb.hi.y : eb.lo.y, (q & 4) ? eb.hi.z : eb.lo.z);
          double h = (c - vec(f.o)).dot(vec(f.z));
          h0 = std::min(h0, h);
          h1 = std::max(h1, h);
        }
      }
      for (double h : {h0, h1}) circle_box(vec(f.o) + vec(f.z) * h, vec(f.z), f.kind == S_CONE ? std::fabs(f.a + h * std::tan(f.b)) : f.a);
    } else if (f.kind == S_SPHERE) {
      bx.add(vec(f.o) - V(f.a, f.a, f.a));
      bx.add(vec(f.o) + V(f.a, f.a, f.a));
    } else if (f.kind == S_TORUS) {
      for (double h : {-f.b, f.b}) circle_box(vec(f.o) + vec(f.z) * h, vec(f.z), f.a + f.b);
    } else {
      for (auto& sp : grids[fi].spans) bx.add(sp.box());
    }
    for (int c = 0; c < 3; c++) f.box[c] = bx.lo[c], f.box[3 + c] = bx.hi[c];
  }
  // ---------------------------------------------------------------- sub-patches
  for (int fi = 0; fi < d->n_faces; fi++) {
    if (P.faces[fi].nurbs < 0) continue;
    const SpanGrid& g = grids[fi];
    for (int a = 0; a < g.nsu; a++)
      for (int b = 0; b < g.nsv; b++) {
        std::vector<std::pair<Bicubic, int>> todo = {{g.spans[a * g.nsv + b], 0}};
        while (!todo.empty()) {
          Bicubic sp = todo.back().first;
          int depth = todo.back().second;
          todo.pop_back();
          DSub s{};
          double rho;
          if (!patch_bounds(sp, &s.sa, &s.sb, &s.lam, s.d2, &rho)) {
            *err = "face " + std::to_string(fi) + ": a weight is not positive";
            return false;
          }
          Bx bx = sp.box();
          s.diag = (bx.hi - bx.lo).len();
          if (rho < need + s.diag && depth < 3) {
            Bicubic l, r, ll, lr, rl, rr;
            sp.split_u(0.5, &l, &r);
            l.split_v(0.5, &ll, &lr);
            r.split_v(0.5, &rl, &rr);
            for (Bicubic* q : {&rr, &rl, &lr, &ll}) todo.push_back({*q, depth + 1});
            continue;
          }
          double plo[2] = {sp.u0, sp.v0}, phi[2] = {sp.u1, sp.v1};
          int klass = trees[fi].box_class(plo, phi);
          if (klass == 0) continue;  // wholly outside its face
          s.face = fi;
          s.nurbs = P.faces[fi].nurbs;
          s.span_a = a;
          s.span_b = b;
          s.klass = klass;
          s.u0 = sp.u0, s.u1 = sp.u1, s.v0 = sp.v0, s.v1 = sp.v1;
          for (auto& c : collapsed[fi]) {
            if (c.k == 0 && sp.u0 == c.value) s.pole_sides |= 1;
            if (c.k == 0 && sp.u1 == c.value) s.pole_sides |= 2;
            if (c.k == 1 && sp.v0 == c.value) s.pole_sides |= 4;
            if (c.k == 1 && sp.v1 == c.value) s.pole_sides |= 8;
          }
          for (int c = 0; c < 3; c++) s.box[c] = bx.lo[c], s.box[3 + c] = bx.hi[c];
          V mid = bx.mid();
          s.c[0] = mid.x, s.c[1] = mid.y, s.c[2] = mid.z;
          P.subs.push_back(s);
          for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
              const H& h = sp.p[i][j];
              P.sub_cp.push_back({h[0], h[1], h[2], h[3]});
              P.sub_cp32.push_back({float(h[0] - mid.x * h[3]), float(h[1] - mid.y * h[3]), float(h[2] - mid.z * h[3]), float(h[3])});
            }
        }
      }
  }
  // ---------------------------------------------------------------- vertices (solid3.rs:797-834)
  std::vector<V> pn(d->n_verts);
  auto tangent_at = [&](int ei, double s) {
    const DEdge& e = P.edges[ei];
    if (e.kind == 0) return (vec(e.b) - vec(e.a)).unit();
    if (e.kind == 1) {
      double t = e.t0 + s * e.sweep;
      return (vec(e.x) * (-std::sin(t)) + vec(e.y) * std::cos(t)) * (e.sweep >= 0 ? 1.0 : -1.0);
    }
    int n = e.n_pieces;
    int k = std::min(int(s * n), n - 1);
    Cubic3 z;
    for (int j = 0; j < 4; j++)
      for (int c = 0; c < 4; c++) z.c[j][c] = P.pieces[e.first_piece + k].cp[j][c];
    V p, d1;
    z.eval(s * n - k, &p, &d1);
    return d1.unit();
  };
  auto face_normal = [&](int fi, V x) {
    const DFace& f = P.faces[fi];
    if (f.kind != S_NURBS) return analytic_normal(f, x);
    double u, v, dist;
    V n;
    nearest_on(grids[fi], x, &u, &v, &n, &dist);
    return n * f.sense;
  };
  for (int fi = 0; fi < d->n_faces; fi++) {
    const IcamFaceDesc& fd = d->faces[fi];
    int k = 0;
    while (k < fd.n_uses) {
      int loop = d->uses[fd.first_use + k].loop, e0 = k;
      while (k < fd.n_uses && d->uses[fd.first_use + k].loop == loop) k++;
      int len = k - e0;
      for (int i = 0; i < len; i++) {
        const IcamUseDesc& ua = d->uses[fd.first_use + e0 + i];
        const IcamUseDesc& ub = d->uses[fd.first_use + e0 + (i + 1) % len];
        int vtx = ua.rev ? d->edges[ua.edge].v0 : d->edges[ua.edge].v1;
        V x(d->verts[3 * vtx], d->verts[3 * vtx + 1], d->verts[3 * vtx + 2]);
        V n = face_normal(fi, x);
        auto use_tan = [&](const IcamUseDesc& u, double s) { return u.rev ? -tangent_at(u.edge, 1.0 - s) : tangent_at(u.edge, s); };
        auto proj = [&](V t) { return (t - n * n.dot(t)).unit(); };
        V ti = proj(use_tan(ua, 1.0)), to = proj(use_tan(ub, 0.0));
        double turn = std::atan2(n.dot(ti.cross(to)), ti.dot(to));
        pn[vtx] = pn[vtx] + n * (PI - turn);
      }
    }
  }
  for (int i = 0; i < d->n_verts; i++) {
    DVert v{};
    for (int k = 0; k < 3; k++) v.p[k] = d->verts[3 * i + k];
    v.pn[0] = pn[i].x, v.pn[1] = pn[i].y, v.pn[2] = pn[i].z;
    P.verts.push_back(v);
  }
  // ---------------------------------------------------------------- poles (solid3.rs:1615-1625)
  // A collapsed side's point at no vertex, with the side's middle inside the face, is a
  // point feature packed after the vertices: its distance and its sign by the fan
  // pseudo-normal (solid3.rs:1960-1986) times the face's sense. Near the point the surface
  // is the cone of its limiting tangents S_k(w), with limiting normals S_k x S_kw (u held)
  // or S_kw x S_v (v held), oriented as S_u x S_v just inside; each pair of neighbouring
  // samples (513 along the side) whose side is covered by the face (the trim tested 1e-9
  // of the domain into it) adds its mean normal times the angle its tangent turns through.
  for (int fi = 0; fi < d->n_faces; fi++)
    for (auto& c : collapsed[fi]) {
      bool at_vertex = false;
      for (int i = 0; i < d->n_verts; i++)
        if ((V(d->verts[3 * i], d->verts[3 * i + 1], d->verts[3 * i + 2]) - c.x).len() <= d->tol) at_vertex = true;
      if (at_vertex) continue;
      const SpanGrid& g = grids[fi];
      double u0, u1, v0, v1;
      grid_domain(g, &u0, &u1, &v0, &v1);
      const double r0 = c.k == 0 ? u0 : v0, r1 = c.k == 0 ? u1 : v1;
      const double o0 = c.k == 0 ? v0 : u0, o1 = c.k == 0 ? v1 : u1;
      auto inside = [&](double along, double w) {
        return c.k == 0 ? trees[fi].inside(along, w) : trees[fi].inside(w, along);
      };
      if (!inside(c.value, 0.5 * (o0 + o1))) continue;
      const double h = c.value == r0 ? 1.0 : -1.0, step = 1e-9 * (r1 - r0) * h;
      const int n = 512;
      V out, ptan, pnrm;
      bool have = false, pcov = false;
      for (int i = 0; i <= n; i++) {
        const double w = o0 + (o1 - o0) * i / double(n);
        V Pp, Ps, Pt, Pst;
        if (c.k == 0)
          grid_eval(g, c.value, w, &Pp, &Ps, &Pt, &Pst);
        else
          grid_eval(g, w, c.value, &Pp, &Ps, &Pt, &Pst);
        const V tan = (c.k == 0 ? Ps : Pt) * h;
        const V nrm = (c.k == 0 ? Ps.cross(Pst) : Pst.cross(Pt)) * h;
        const bool cov = inside(c.value + step, w);
        if (have && pcov && cov && tan.len() > 0.0 && ptan.len() > 0.0) {
          const V ta = ptan.unit(), tb = tan.unit();
          const double ang = std::atan2(ta.cross(tb).len(), ta.dot(tb));
          const V m = pnrm.unit() + nrm.unit();
          if (m.len() > 0.0) out = out + m.unit() * ang;
        }
        ptan = tan, pnrm = nrm, pcov = cov, have = true;
      }
      const V fn = out * P.faces[fi].sense;
      DVert v{};
      v.p[0] = c.x.x, v.p[1] = c.x.y, v.p[2] = c.x.z;
      v.pn[0] = fn.x, v.pn[1] = fn.y, v.pn[2] = fn.z;
      P.verts.push_back(v);
    }
  // ---------------------------------------------------------------- the tree over every feature
  std::vector<Item> items;
  Bx all;
  auto box6 = [](const double* b) {
    Bx x;
    x.add(V(b[0], b[1], b[2]));
    x.add(V(b[3], b[4], b[5]));
    return x;
  };
  for (int i = 0; i < int(P.faces.size()); i++)
    if (P.faces[i].kind != S_NURBS) items.push_back({(uint32_t(IK_FACE) << IK_SHIFT) | uint32_t(i), box6(P.faces[i].box)});
  for (int i = 0; i < int(P.subs.size()); i++) items.push_back({(uint32_t(IK_SUB) << IK_SHIFT) | uint32_t(i), box6(P.subs[i].box)});
  for (int i = 0; i < int(P.edges.size()); i++)
    if (P.edges[i].kind <= 1) items.push_back({(uint32_t(IK_EDGE) << IK_SHIFT) | uint32_t(i), box6(P.edges[i].box)});
  for (int i = 0; i < int(P.pieces.size()); i++) items.push_back({(uint32_t(IK_PIECE) << IK_SHIFT) | uint32_t(i), box6(P.pieces[i].box)});
  for (int i = 0; i < int(P.verts.size()); i++) {
    Bx b;
    b.add(V(P.verts[i].p[0], P.verts[i].p[1], P.verts[i].p[2]));
    items.push_back({(uint32_t(IK_VERT) << IK_SHIFT) | uint32_t(i), b});
  }
  for (auto& it : items) all.add(it.box);
  for (int k = 0; k < 3; k++) P.lo[k] = all.lo[k], P.hi[k] = all.hi[k];
  P.bvh.assign(1, DBvh{});
  build_bvh(items, 0, int(items.size()), 0, P.bvh, P.items);
  return true;
}

}  // namespace icam
