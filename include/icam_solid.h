/*
 * icam_solid.h — the solid description handed across the C ABI.
 *
 * A closed manifold B-rep as the reference's import produces it
 * (crates/icam-core/src/solid3.rs:39-278: Face3, EdgeRec, Vert, Use), flattened
 * into plain arrays so that a Rust, C or Python host can fill it without any
 * type of this library:
 *
 *  - faces: one surface each (plane, cylinder, cone, sphere, torus in their STEP
 *    parametrisations, surface3.rs:1-12; or a rational B-spline given as its grid
 *    of Bezier spans, surface3.rs:1150-1160), the outward sense, the parameter
 *    domain its trim loops live in, and its loop uses;
 *  - edges: line, circular arc, or a rational B-spline as Bezier pieces
 *    (curve3.rs:489-498), with the two faces that use it (the same face twice
 *    for a seam);
 *  - uses: one edge use of a face loop with its parameter-domain curve (the
 *    "pcurve", trim2.rs:40-62), as rational cubic Bezier pieces in (u, v).
 *
 * Analytic faces' parameters follow Analytic::uv (trim2.rs:1904-1933) except
 * that the angular parameter is the angle itself (radians, period 2 pi) rather
 * than the quarter-arc parameter: a face's loops and its uv map only have to
 * agree with each other.
 *
 * Units: millimetres. Homogeneous points are (x w, y w, z w, w) with w > 0.
 */
#ifndef ICAM_SOLID_H
#define ICAM_SOLID_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Surface kinds (surface3.rs:24-35). */
enum {
  ICAM_PLANE = 0,
  ICAM_CYLINDER = 1,
  ICAM_CONE = 2,
  ICAM_SPHERE = 3,
  ICAM_TORUS = 4,
  ICAM_NURBS = 5
};

/* Edge curve kinds (curve3.rs:489-498; ellipses are not produced here). */
enum { ICAM_EDGE_LINE = 0, ICAM_EDGE_ARC = 1, ICAM_EDGE_SPLINE = 2 };

/* A right-handed frame: origin, unit z axis, unit x axis (y = z cross x). */
typedef struct IcamFrame {
  double o[3];
  double z[3];
  double x[3];
} IcamFrame;

typedef struct IcamFaceDesc {
  int32_t kind;  /* ICAM_PLANE .. ICAM_NURBS */
  int32_t sense; /* +1 when the outward normal is the surface's own normal */
  IcamFrame f;   /* analytic surfaces */
  /* cylinder: a = r; cone: a = r at height 0, b = semi-angle (rad);
   * sphere: a = r; torus: a = major, b = minor. */
  double a, b;
  /* B-spline faces: degrees, spans along u and v; Bezier control points of
   * span (i, j) start at patches[patch_off + (i * nsv + j) * (du+1)*(dv+1)*4],
   * point (k, l) (k along u) at + (k * (dv+1) + l) * 4; the span breakpoints are
   * breaks[brk_off .. + nsu] (u) then breaks[brk_off + nsu + 1 .. + nsv] (v). */
  int32_t du, dv, nsu, nsv;
  int64_t patch_off;
  int64_t brk_off;
  /* The parameter domain of the trim loops and each direction's period
   * (0 when not periodic). */
  double lo[2], hi[2], period[2];
  /* This face's loop uses: uses[first_use .. first_use + n_uses), loop by loop,
   * each loop in traversal order. */
  int32_t first_use, n_uses;
} IcamFaceDesc;

typedef struct IcamEdgeDesc {
  int32_t kind;   /* ICAM_EDGE_LINE, ICAM_EDGE_ARC, ICAM_EDGE_SPLINE */
  int32_t v0, v1; /* start and end vertex in the stored direction */
  int32_t f0, f1; /* the faces using it (f0 == f1 for a seam) */
  /* splines: degree and pieces[first_piece ..+ n_pieces] in cpieces, each
   * (degree+1) homogeneous points, in the stored direction */
  int32_t degree, first_piece, n_pieces;
  int32_t pad;
  double a[3], b[3]; /* line ends */
  IcamFrame f;       /* arc: P(t) = o + r (cos t x + sin t y), t = t0 .. t0 + sweep */
  double r, t0, sweep;
} IcamEdgeDesc;

typedef struct IcamUseDesc {
  int32_t edge;
  int32_t rev;  /* the loop runs against the edge's stored direction */
  int32_t loop; /* loop index within the face */
  int32_t seam; /* the face uses this edge twice: not a boundary of it */
  /* the use's curve in the face's (u, v), in traversal order: n_pc rational
   * cubic Bezier pieces in pcurves, 12 doubles each: 4 x (u w, v w, w) */
  int32_t first_pc, n_pc;
} IcamUseDesc;

typedef struct IcamSolidDesc {
  int32_t n_faces, n_edges, n_verts, n_uses;
  const IcamFaceDesc* faces;
  const IcamEdgeDesc* edges;
  const double* verts; /* n_verts x 3 */
  const IcamUseDesc* uses;
  const double* patches;
  const double* breaks;
  const double* cpieces;
  const double* pcurves;
  int64_t n_patch_doubles, n_break_doubles, n_cpiece_doubles, n_pcurve_doubles;
  double tol; /* model tolerance (mm) */
} IcamSolidDesc;

#ifdef __cplusplus
}
#endif

#endif /* ICAM_SOLID_H */
