// Device layout of a packed solid: structure-of-arrays records by feature kind, the
// trim trees of every face, the B-spline faces' spans and certified sub-patches, and
// one bounding-volume tree over every feature for culling. Plain structs shared by
// the host builder (pack_build.cpp) and the kernels; every record is 8-byte aligned.
//
// The reference packs the same evaluator into word arrays for its WGSL kernel
// (crates/icam-core/src/solid3/gpu.rs:259-701: FACE, EDGE, VERT, SUB, CURVE records);
// here each kind keeps its own array of fixed-size records in HBM, doubles for the
// exact path and a rebased float copy of the control nets for the mixed path.
#pragma once

#include <cstdint>

#include <vector_types.h>

namespace icam {

// Feature codes: kind << 28 | index (the reference's candidate codes, gpu.rs:705-731).
enum ItemKind : uint32_t { IK_FACE = 0, IK_SUB = 1, IK_EDGE = 2, IK_PIECE = 3, IK_VERT = 4 };
constexpr uint32_t IK_SHIFT = 28;
constexpr uint32_t IK_MASK = (1u << IK_SHIFT) - 1;

enum SurfKind : int32_t { S_PLANE = 0, S_CYLINDER = 1, S_CONE = 2, S_SPHERE = 3, S_TORUS = 4, S_NURBS = 5 };

struct DFace {
  int32_t kind;
  int32_t trim;    // root cell of its trim tree; -1: no loop pieces (the whole surface)
  int32_t nurbs;   // index into the B-spline face table, or -1
  int32_t pad;
  double sense;    // +1 / -1
  double o[3], z[3], x[3], y[3];
  double a, b;
  double lo[2], hi[2], period[2];  // trim domain
  double box[6];                   // face_box (solid3.rs:1211-1278)
};

// A B-spline face: its grid of bicubic spans (spans[first_span + a * nsv + b]).
struct DNurbs {
  int32_t face, first_span, nsu, nsv;
  int32_t first_break;  // breaks[first_break .. + nsu] (u) then (.. + nsv) (v)
  int32_t pad;
};

// A certified sub-patch of a B-spline span, always bicubic rational: its control
// points are cp[16 * index + 4 * i + j] (i along u), homogeneous doubles, and
// cp32[...] the same rebased to `c` in floats.
struct DSub {
  int32_t face, nurbs, span_a, span_b;
  int32_t klass;  // trim class of its parameter rectangle: 1 wholly inside, -1 straddles
  // its sides on a side of the face's domain that the surface collapses on to one point
  // (a pole): bit 0 s = 0, 1 s = 1, 2 t = 0, 3 t = 1; a part of it touching one is never
  // cleared by the critical-point test (surface3.rs:579-591 Creases)
  int32_t pole_sides;
  double u0, u1, v0, v1;  // its rectangle in the face's parameters
  double box[6];          // control-point box
  double c[3];            // rebasing origin (box centre)
  double diag;
  // Convexity certificate (surface3.rs:814-925, restated): parameters scaled so both
  // tangents have unit length at the middle (sa, sb); lam a lower bound of
  // lambda_min(G) over the sub-patch; d2 the intervals of S_ss, S_st, S_tt per
  // component, [k][comp][lo,hi].
  double sa, sb, lam;
  double d2[3][3][2];
};

struct DEdge {
  int32_t kind;  // 0 line, 1 arc, 2 spline, 3 a crease of face f0 (= f1) inside it
  int32_t f0, f1;
  int32_t first_piece, n_pieces;
  int32_t pad;
  double a[3], b[3];
  double o[3], z[3], x[3], y[3];
  double r, t0, sweep;
  double box[6];
};

// A flat piece of a spline edge (curve3.rs:345-372): a rational cubic in 3D.
struct DPiece {
  int32_t edge;
  int32_t first, last;  // first / last piece of its edge (its ends are the edge's)
  int32_t pad;
  double cp[4][4];
  double box[6];
  double thick;
  double lam;           // lower bound of |C'|^2 over the piece
  double d2[3][2];      // interval of C'' per component
  // For each adjacent face that is a B-spline face: its parameters at the piece's two
  // ends (a seed for the normal there; -1 span when the face is analytic).
  double uv[2][2][2];   // [side][end][u,v]
};

// A point feature with its pseudo-normal: the solid's vertices (angle-weighted), then
// its B-spline faces' poles (a collapsed side's point, the fan pseudo-normal).
struct DVert {
  double p[3];
  double pn[3];
};

// A trim cell (trim2.rs:66-94): low and high corners, its reference point and the
// answer there, its kind (0 leaf, 1 crossed, 2 split), the instance list (crossed) or
// the four children (split; child k = (u >= mid u) + 2 (v >= mid v)).
struct DCell {
  double lo[2], hi[2], r[2];
  int32_t inside, kind, first, count;
  int32_t kids[4];
};

// A shifted copy of a loop piece (periodic directions).
struct DInst {
  int32_t piece, pad;
  double shift[2];
};

// One node of the bounding-volume tree: leaf when count > 0 (items[first .. +count]),
// else children left = first, right = first + 1.
struct DBvh {
  float lo[3], hi[3];
  int32_t first, count;
};

// Everything the kernels read, by device pointer.
struct DPack {
  const DFace* faces;
  const DNurbs* nurbs;
  const DSub* subs;
  const double4* sub_cp;
  const float4* sub_cp32;
  const double4* span_cp;  // spans of every B-spline face, bicubic
  const double* breaks;
  const DEdge* edges;
  const DPiece* pieces;
  const DVert* verts;
  const DCell* cells;
  const DInst* insts;
  const int32_t* among;    // instance lists of crossed cells
  const double* tpieces;   // loop pieces, 12 doubles each: 4 x (u w, v w, w)
  const DBvh* bvh;
  const uint32_t* items;   // bvh leaves' feature codes
  int32_t n_faces, n_subs, n_edges, n_pieces, n_verts, n_bvh, n_items;
  int32_t pad;
  double tol;
  double lo[3], hi[3];     // the part's box
};

}  // namespace icam
