// The host-side image of a packed solid (pack.h records in host vectors) and its builder.
#pragma once

#include <string>
#include <vector>

#include <vector_types.h>

#include "../../include/icam_solid.h"
#include "host_geom.h"
#include "pack.h"

namespace icam {

struct HostPack {
  std::vector<DFace> faces;
  std::vector<DNurbs> nurbs;
  std::vector<DSub> subs;
  std::vector<double4> sub_cp;
  std::vector<float4> sub_cp32;
  std::vector<double4> span_cp;
  std::vector<double> breaks;
  std::vector<DEdge> edges;
  std::vector<DPiece> pieces;
  std::vector<DVert> verts;
  std::vector<DCell> cells;
  std::vector<DInst> insts;
  std::vector<int32_t> among;
  std::vector<double> tpieces;
  std::vector<DBvh> bvh;
  std::vector<uint32_t> items;
  double tol = 1e-9;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

// Packs a solid; `need` is the distance within which B-spline sub-patches should
// certify convexity (they are split until they do, or 3 levels deep).
bool build_pack(const IcamSolidDesc* d, double need, HostPack* out, std::string* err);

}  // namespace icam
